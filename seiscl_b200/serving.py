"""Modelling service: a queue of forward / gradient requests served by a pool
of workers sharing one GPU.

Requests are taken from one FIFO queue as soon as a worker is free and the
request's device-memory footprint fits in the service's budget (continuous
batching at request granularity: a request arriving while others run is
admitted as a worker and memory free up).  A running request holds a plan
-- its own device buffers and CUDA stream, its time loops captured as CUDA
graphs -- and the shots of a 2D request advance together in that plan
(``Config.batch``: one launch per kernel and time step for all of them), so
that small grids fill the GPU; requests of different workers run
concurrently on their own streams.  Optionally (``max_slots``) the shots of
other requests are spread over several plans that run at the same time.
Finished plans stay in a shared cache for the next request with the same
configuration.

A request's result depends only on the request: every shot starts from
zeroed wave fields on a plan whose model is set from the request; the batch,
the number of slots and the shot-to-slot assignment depend only on the
request; per-shot gradient copies are summed in a fixed order; so the output
is the same whatever else is in flight (tested).

This is the serving layer SeisCL does not have (SeisCL runs one job per
process, src/SeisCL_MPI.c); the per-shot work is the same forward and adjoint
path as ``Plan.forward`` / ``Plan.adjoint``.
"""
from __future__ import annotations

import collections
import dataclasses
import queue
import threading
import time
from concurrent.futures import Future
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import engine


@dataclasses.dataclass
class Request:
    """One job: a grid configuration, its model and its shots.

    ``model``: dict with vp, vs, rho[, taup, taus] in engine host layout
    ([nx][(ny)][nz]).  ``shots``: list of (src_pos [nsrc][5], src [nsrc][NT],
    rec_pos [nrec][8]).  ``kind``: "forward" (seismograms of ``outputs``) or
    "gradient" (L2 misfit against ``observed``, one [nrec][NT] array per
    output and shot, and the summed parameter gradient)."""
    config: engine.Config
    model: Dict[str, np.ndarray]
    shots: Sequence[Tuple[np.ndarray, np.ndarray, np.ndarray]]
    outputs: Sequence[str] = ("vx", "vz")
    kind: str = "forward"
    observed: Optional[Sequence[Dict[str, np.ndarray]]] = None
    rid: int = 0


@dataclasses.dataclass
class Result:
    rid: int
    seismograms: List[Dict[str, np.ndarray]]
    gradient: Optional[Dict[str, np.ndarray]]
    misfit: float
    t_submit: float
    t_start: float
    t_done: float

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


def _key(cfg: engine.Config):
    return tuple((f.name, repr(getattr(cfg, f.name))) for f in dataclasses.fields(cfg))


CHECKPOINT_STEPS = 50   # snapshot interval of viscoelastic gradient requests


def plan_config(req: Request, max_batch: int = 8, batch_bytes: int = 24 << 30) -> engine.Config:
    """The configuration of the plans serving ``req``: several shots of a
    request advance together in one plan (``batch``: up to ``max_batch``
    shots, as many as fit in ``batch_bytes`` of device memory; P-SV,
    acoustic forward and 3D requests with FP32 fields).  A function of the
    request alone."""
    c = req.config
    n = len(req.shots)
    if req.kind == "gradient" and c.L > 0 and c.ND in (2, 3) and c.back_prop_type != 2 and not c.checkpoint:
        # with memory variables the backpropagation from saved boundaries
        # (the reference's BACK_PROP_TYPE 1) is unstable over long runs: the
        # forward field is recomputed from snapshots instead, one shot per launch
        return dataclasses.replace(c, checkpoint=CHECKPOINT_STEPS)
    ok = (c.ND in (2, 3) or (c.ND == 22 and req.kind == "forward")) and c.back_prop_type != 2 and \
        c.field_precision == "fp32" and c.kernels in ("fast", "general", "stream", "vector") and not c.checkpoint
    if n < 2 or max_batch < 2 or not ok:
        return c
    b = min(n, max_batch)
    while b > 1 and request_footprint(req, dataclasses.replace(c, batch=b)) > batch_bytes:
        b -= 1
    return dataclasses.replace(c, batch=b) if b > 1 else c


def request_footprint(req: Request, cfg: Optional[engine.Config] = None, max_batch: int = 8) -> int:
    """Device bytes one plan serving ``req`` holds: model, wave fields, CPML
    memory and shot buffers, plus saved boundaries, adjoint fields and
    gradient sums for a gradient request (``engine.footprint``), for the
    plan configuration ``cfg`` (default: ``plan_config(req)``)."""
    cfg = cfg or plan_config(req, max_batch)
    per = max(1, cfg.batch)
    nsrc = sorted((np.asarray(sp).reshape(-1, 5).shape[0] for sp, _, _ in req.shots), reverse=True)
    nrec = sorted((np.asarray(rp).reshape(-1, 8).shape[0] for _, _, rp in req.shots), reverse=True)
    return engine.footprint(cfg, req.kind == "gradient", max(1, sum(nsrc[:per])), sum(nrec[:per]) * len(req.outputs),
                            len(cfg.gradfreqs))


def shot_slots(req: Request, footprint: int, max_slots: int = 1, slot_bytes: int = 1 << 30,
               max_batch: int = 8) -> int:
    """Plans a request's shots are spread over: up to ``max_slots`` for
    grids whose plan needs at most ``slot_bytes``, else one; batched plans
    take one slot.  A function of the request alone, so its result does not
    depend on the load."""
    if footprint > slot_bytes or plan_config(req, max_batch).batch > 1:
        return 1
    return max(1, min(len(req.shots), max_slots))


def serve(plans, req: Request) -> Result:
    """Run one request on ``plans`` (one plan or a list; synchronously).
    Shot i runs on plan i % len(plans); the plans run at the same time."""
    if not isinstance(plans, (list, tuple)):
        plans = [plans]
    k = len(plans)
    if req.kind not in ("forward", "gradient"):
        raise ValueError("unknown request kind %r" % req.kind)
    if req.kind == "gradient" and (req.observed is None or len(req.observed) != len(req.shots)):
        raise ValueError("a gradient request needs observed data for every shot")
    m = req.model
    n = len(req.shots)
    seis: List[Optional[Dict[str, np.ndarray]]] = [None] * n
    misfits = [0.0] * n
    grads: List[Optional[Dict[str, np.ndarray]]] = [None] * k

    def run_slot(j):
        plan = plans[j]
        B = max(1, int(getattr(plan.cfg, "batch", 1)))
        plan.set_model(m["vp"], m.get("vs"), m["rho"], m.get("taup"), m.get("taus"))
        if req.kind == "gradient":
            plan.zero_gradient()
        mine = list(range(j, n, k))
        for g0 in range(0, len(mine), B):
            idx = mine[g0:g0 + B]
            group = [req.shots[i] for i in idx]
            grad = req.kind == "gradient"
            if B > 1:
                ds = plan.forward_batch(group, list(req.outputs), save_boundaries=grad)
            else:
                sp, src, rp = group[0]
                ds = [plan.forward(sp, src, rp, list(req.outputs), save_boundaries=grad)]
            adj = []
            for i, d in zip(idx, ds):
                seis[i] = d
                if not grad:
                    continue
                res = {o: d[o] - np.asarray(req.observed[i][o], np.float32) for o in req.outputs}
                misfits[i] = sum(float((r.astype(np.float64) ** 2).sum()) for r in res.values())
                adj.append(plan.residual_scale(req.shots[i][2], res))
            if grad:
                if B > 1:
                    plan.adjoint_batch(group, adj)
                else:
                    sp, src, rp = group[0]
                    plan.adjoint(sp, src, rp, adj[0])
        if req.kind == "gradient":
            grads[j] = plan.gradient(transform=True)

    if k == 1:
        run_slot(0)
    else:
        errors: List[BaseException] = []

        def guarded(j):
            try:
                run_slot(j)
            except BaseException as exc:  # re-raised below
                errors.append(exc)

        threads = [threading.Thread(target=guarded, args=(j,), name="sfd-slot-%d" % j) for j in range(k)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]
    grad = None
    if req.kind == "gradient":
        if k == 1:
            grad = grads[0]
        else:   # the chain rule is linear in the accumulated kernels: sum in slot order
            grad = {name: np.sum([g[name].astype(np.float64) for g in grads], axis=0).astype(np.float32)
                    for name in grads[0]}
        vs = m.get("vs")
        if vs is not None and not np.any(vs):
            # acoustic media run as P-SV with vs = 0: the vs gradient carries
            # 1 / mu^2 and is undefined; vp and rho are the acoustic gradient
            grad.pop("vs", None)
    return Result(req.rid, seis, grad, float(sum(misfits)), 0.0, 0.0, 0.0)


def serve_alone(req: Request, max_slots: int = 1, slot_bytes: int = 1 << 30,
                footprint=request_footprint, max_batch: int = 8) -> Result:
    """The request on fresh plans, with the configuration and slots a
    ``Server`` with the same settings would give it (the reference for
    results in a mix)."""
    k = shot_slots(req, int(footprint(req)), max_slots, slot_bytes, max_batch)
    plans = [engine.Plan(plan_config(req, max_batch)) for _ in range(k)]
    try:
        return serve(plans, req)
    finally:
        for p in plans:
            p.close()


class Server:
    """``Server(workers=8)``; ``submit(request) -> Future[Result]``;
    ``close()`` drains the queue and stops the workers.

    Admission by device memory: every plan the service holds (running or
    idle in the shared plan cache) is counted at its footprint
    (``request_footprint``) against ``memory_budget`` (bytes; default 90 %
    of the device's free memory when the first request is admitted).
    Requests are admitted in arrival order as soon as a worker is free and
    the footprint of their slots fits; idle cached plans are evicted (least
    recently used first) to make room, and otherwise the request waits for
    running ones to finish.  A request larger than the whole budget fails
    with MemoryError.  Up to ``workers * plans_per_worker`` idle plans are
    kept, so a configuration seen again reuses its device buffers and
    captured loops.  ``max_batch``: see ``plan_config``; ``max_slots`` /
    ``slot_bytes``: see ``shot_slots``."""

    def __init__(self, workers: int = 8, plans_per_worker: int = 4, device: Optional[int] = None,
                 memory_budget: Optional[int] = None, footprint=request_footprint, max_slots: int = 1,
                 slot_bytes: int = 1 << 30, max_batch: int = 8):
        self._q: "queue.Queue" = queue.Queue()
        self._closed = False
        self._device = device
        self._footprint = footprint
        self._budget = memory_budget
        self._max_slots = max_slots
        self._slot_bytes = slot_bytes
        self._max_batch = max_batch
        self._max_idle = max(1, workers * plans_per_worker)
        self._cv = threading.Condition()
        self._idle: "collections.OrderedDict" = collections.OrderedDict()  # id -> (key, plan, bytes)
        self._held = 0          # bytes of every plan alive (running and idle)
        self._tickets = 0       # next arrival number
        self._next_admit = 0    # arrival number admitted next
        self._stats = {"admitted": 0, "rejected": 0, "evicted": 0, "waited": 0, "peak_bytes": 0, "slots": 0}
        self._threads = [threading.Thread(target=self._run, name="sfd-worker-%d" % i, daemon=True)
                         for i in range(workers)]
        for t in self._threads:
            t.start()

    def submit(self, req: Request) -> Future:
        if self._closed:
            raise RuntimeError("server closed")
        fut: Future = Future()
        with self._cv:
            ticket = self._tickets
            self._tickets += 1
            self._q.put((req, fut, time.perf_counter(), ticket))
        return fut

    def close(self):
        self._closed = True
        for _ in self._threads:
            self._q.put(None)
        for t in self._threads:
            t.join()
        with self._cv:
            for _, plan, _ in self._idle.values():
                plan.close()
            self._idle.clear()
        if self._budget is not None and self._footprint is request_footprint:
            # give the device memory of the closed plans back, on the
            # service's device (a thread, so the caller's device is untouched)
            def release():
                try:
                    if self._device is not None:
                        import torch

                        torch.cuda.set_device(self._device)
                    engine.release_memory()
                except Exception:
                    pass

            t = threading.Thread(target=release)
            t.start()
            t.join()

    def stats(self) -> Dict[str, int]:
        """Admission counters, the budget and the peak of bytes held."""
        with self._cv:
            return dict(self._stats, budget=self._budget or 0, held=self._held)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------ admission
    def _skip(self, ticket: int):
        with self._cv:
            while self._next_admit != ticket:
                self._cv.wait()
            self._next_admit += 1
            self._cv.notify_all()

    def _admit(self, ticket: int, key, need: int, k: int):
        """Wait for this request's turn and room for k plans of ``need``
        bytes; returns [(cached plan or None, bytes it will hold)] * k."""
        with self._cv:
            while self._next_admit != ticket:
                self._cv.wait()
            try:
                if self._budget is None:
                    self._budget = int(0.9 * engine.device_memory()[0])
                if k * need > self._budget:
                    self._stats["rejected"] += 1
                    raise MemoryError("request needs %d bytes of device memory; the service budget is %d"
                                      % (k * need, self._budget))
                waited = False
                while True:
                    mine = [i for i, (kk, _, _) in self._idle.items() if kk == key][:k]
                    extra = sum(max(0, need - self._idle[i][2]) for i in mine) + (k - len(mine)) * need
                    if self._held + extra <= self._budget:
                        break
                    victim = next((i for i in self._idle if i not in mine), None)
                    if victim is not None:
                        _, vplan, vbytes = self._idle.pop(victim)
                        vplan.close()
                        self._held -= vbytes
                        self._stats["evicted"] += 1
                        continue
                    waited = True
                    self._cv.wait()
                out = []
                for i in mine:
                    _, plan, have = self._idle.pop(i)
                    out.append((plan, max(have, need)))
                out += [(None, need)] * (k - len(mine))
                self._held += extra
                self._stats["admitted"] += 1
                self._stats["slots"] += k
                self._stats["waited"] += int(waited)
                self._stats["peak_bytes"] = max(self._stats["peak_bytes"], self._held)
                return out
            finally:
                self._next_admit += 1
                self._cv.notify_all()

    def _release(self, key, held):
        with self._cv:
            for plan, nbytes in held:
                if plan is None:
                    self._held -= nbytes
                    continue
                self._idle[id(plan)] = (key, plan, nbytes)
            while len(self._idle) > self._max_idle:
                _, (_, vplan, vbytes) = self._idle.popitem(last=False)
                vplan.close()
                self._held -= vbytes
                self._stats["evicted"] += 1
            self._cv.notify_all()

    # ------------------------------------------------------------ worker
    def _run(self):
        if self._device is not None:
            import torch

            torch.cuda.set_device(self._device)
        while True:
            item = self._q.get()
            if item is None:
                return
            req, fut, t_submit, ticket = item
            cfg = plan_config(req, self._max_batch)
            key = _key(cfg)
            try:
                need = int(self._footprint(req) if self._footprint is not request_footprint
                           else request_footprint(req, cfg))
                k = shot_slots(req, need, self._max_slots, self._slot_bytes, self._max_batch)
            except BaseException as exc:
                self._skip(ticket)
                fut.set_exception(exc)
                continue
            try:
                held = self._admit(ticket, key, need, k)
            except BaseException as exc:
                fut.set_exception(exc)
                continue
            if not fut.set_running_or_notify_cancel():
                self._release(key, held)
                continue
            t_start = time.perf_counter()
            live = []   # cached plans come first in `held`; new ones are created here
            try:
                for plan, nbytes in held:
                    live.append((plan if plan is not None else engine.Plan(cfg), nbytes))
                res = serve([plan for plan, _ in live], req)
                res.t_submit, res.t_start, res.t_done = t_submit, t_start, time.perf_counter()
                fut.set_result(res)
            except BaseException as exc:  # reported through the future
                fut.set_exception(exc)
            finally:
                self._release(key, live + held[len(live):])


def percentiles(latencies: Sequence[float], qs=(50, 99)) -> Dict[str, float]:
    a = np.sort(np.asarray(latencies, np.float64))
    return {"p%d" % q: float(np.percentile(a, q)) if len(a) else float("nan") for q in qs}


class Router:
    """Requests over several GPUs of one process: one ``Server`` per device
    (its workers bound to that device), each request sent to the server
    with the fewest requests in flight (ties: the first).  The serving
    router across GPUs; ``bench.py --workload serving`` under torchrun runs
    one server per rank instead, each taking its share of the stream.

    ``Router(devices=[0, 1, 2, 3], workers=4, ...)``; other keywords go to
    every ``Server``."""

    def __init__(self, devices: Sequence[Optional[int]], **server_kw):
        if not devices:
            raise ValueError("a router needs at least one device")
        self.devices = list(devices)
        self.servers = [Server(device=d, **server_kw) for d in self.devices]
        self._inflight = [0] * len(self.servers)
        self._lock = threading.Lock()

    def submit(self, req: Request) -> Future:
        with self._lock:
            i = min(range(len(self.servers)), key=lambda k: (self._inflight[k], k))
            self._inflight[i] += 1
        fut = self.servers[i].submit(req)

        def done(_f, i=i):
            with self._lock:
                self._inflight[i] -= 1

        fut.add_done_callback(done)
        return fut

    def stats(self) -> List[Dict[str, int]]:
        return [s.stats() for s in self.servers]

    def close(self):
        for s in self.servers:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
