"""Modelling service: a queue of forward / gradient requests served by a pool
of workers sharing one GPU.

Requests are taken from one FIFO queue as soon as a worker is free and the
request's device-memory footprint fits in the service's budget (continuous
batching at request granularity: a request arriving while others run is
admitted as a worker and memory free up).  Each running request has its own
plan -- its own device buffers and CUDA stream, with its time loops captured
as CUDA graphs -- so small grids from different requests run concurrently on
the GPU while a large one occupies a single worker; finished plans stay in a
shared cache for the next request with the same configuration.  A request's
result depends only on the request: every shot starts from zeroed wave
fields on a plan whose model is set from the request, so the output is the
same whatever else is in flight (tested).

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


def request_footprint(req: Request) -> int:
    """Device bytes the plan serving ``req`` holds: model, wave fields, CPML
    memory and shot buffers, plus saved boundaries, adjoint fields and
    gradient sums for a gradient request (``engine.footprint``)."""
    nsrc = max((np.asarray(sp).reshape(-1, 5).shape[0] for sp, _, _ in req.shots), default=1)
    nrec = max((np.asarray(rp).reshape(-1, 8).shape[0] for _, _, rp in req.shots), default=0)
    return engine.footprint(req.config, req.kind == "gradient", nsrc, nrec * len(req.outputs),
                            len(req.config.gradfreqs))


class Server:
    """``Server(workers=4)``; ``submit(request) -> Future[Result]``;
    ``close()`` drains the queue and stops the workers.

    Admission by device memory: every plan the service holds (running or
    idle in the shared plan cache) is counted at its footprint
    (``request_footprint``) against ``memory_budget`` (bytes; default 90 %
    of the device's free memory when the first request is admitted).
    Requests are admitted in arrival order as soon as a worker is free and
    the footprint fits; idle cached plans are evicted (least recently used
    first) to make room, and otherwise the request waits for running ones to
    finish.  A request larger than the whole budget fails with MemoryError.
    Up to ``workers * plans_per_worker`` idle plans are kept, so a
    configuration seen again reuses its device buffers and captured loops."""

    def __init__(self, workers: int = 4, plans_per_worker: int = 4, device: Optional[int] = None,
                 memory_budget: Optional[int] = None, footprint=request_footprint):
        self._q: "queue.Queue" = queue.Queue()
        self._closed = False
        self._device = device
        self._footprint = footprint
        self._budget = memory_budget
        self._max_idle = max(1, workers * plans_per_worker)
        self._cv = threading.Condition()
        self._idle: "collections.OrderedDict" = collections.OrderedDict()  # id -> (key, plan, bytes)
        self._held = 0          # bytes of every plan alive (running and idle)
        self._tickets = 0       # next arrival number
        self._next_admit = 0    # arrival number admitted next
        self._stats = {"admitted": 0, "rejected": 0, "evicted": 0, "waited": 0, "peak_bytes": 0}
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

    def stats(self) -> Dict[str, int]:
        """Admission counters, the budget and the peak of bytes held."""
        with self._cv:
            return dict(self._stats, budget=self._budget or 0, held=self._held)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------ admission
    def _admit(self, ticket: int, key, need: int):
        """Wait for this request's turn and room for ``need`` bytes; returns
        (cached plan or None, bytes the plan will hold)."""
        with self._cv:
            while self._next_admit != ticket:
                self._cv.wait()
            try:
                if self._budget is None:
                    self._budget = int(0.9 * engine.device_memory()[0])
                if need > self._budget:
                    self._stats["rejected"] += 1
                    raise MemoryError("request needs %d bytes of device memory; the service budget is %d"
                                      % (need, self._budget))
                mine = next((i for i, (k, _, _) in self._idle.items() if k == key), None)
                have = self._idle[mine][2] if mine is not None else 0
                extra = max(0, need - have)
                waited = False
                while self._held + extra > self._budget:
                    victim = next((i for i in self._idle if i != mine), None)
                    if victim is not None:
                        _, vplan, vbytes = self._idle.pop(victim)
                        vplan.close()
                        self._held -= vbytes
                        self._stats["evicted"] += 1
                        continue
                    waited = True
                    self._cv.wait()
                plan = None
                if mine is not None:
                    _, plan, _ = self._idle.pop(mine)
                self._held += extra
                self._stats["admitted"] += 1
                self._stats["waited"] += int(waited)
                self._stats["peak_bytes"] = max(self._stats["peak_bytes"], self._held)
                return plan, have + extra
            finally:
                self._next_admit += 1
                self._cv.notify_all()

    def _release(self, key, plan, nbytes: int):
        with self._cv:
            if plan is None:
                self._held -= nbytes
            else:
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
            key = _key(req.config)
            try:
                need = int(self._footprint(req))
            except BaseException as exc:
                need, plan, nbytes = None, None, 0
                with self._cv:   # keep the arrival order moving
                    while self._next_admit != ticket:
                        self._cv.wait()
                    self._next_admit += 1
                    self._cv.notify_all()
                fut.set_exception(exc)
                continue
            try:
                plan, nbytes = self._admit(ticket, key, need)
            except BaseException as exc:
                fut.set_exception(exc)
                continue
            if not fut.set_running_or_notify_cancel():
                self._release(key, plan, nbytes)
                continue
            t_start = time.perf_counter()
            try:
                if plan is None:
                    plan = engine.Plan(req.config)
                res = serve(plan, req)
                res.t_submit, res.t_start, res.t_done = t_submit, t_start, time.perf_counter()
                fut.set_result(res)
            except BaseException as exc:  # reported through the future
                fut.set_exception(exc)
            finally:
                self._release(key, plan, nbytes)


def serve(plan, req: Request) -> Result:
    """Run one request on ``plan`` (synchronously)."""
    m = req.model
    plan.set_model(m["vp"], m.get("vs"), m["rho"], m.get("taup"), m.get("taus"))
    seis = []
    misfit = 0.0
    grad = None
    if req.kind == "forward":
        for sp, src, rp in req.shots:
            seis.append(plan.forward(sp, src, rp, list(req.outputs)))
    elif req.kind == "gradient":
        if req.observed is None or len(req.observed) != len(req.shots):
            raise ValueError("a gradient request needs observed data for every shot")
        plan.zero_gradient()
        for (sp, src, rp), obs in zip(req.shots, req.observed):
            d = plan.forward(sp, src, rp, list(req.outputs), save_boundaries=True)
            seis.append(d)
            res = {k: d[k] - np.asarray(obs[k], np.float32) for k in req.outputs}
            misfit += sum(float((r.astype(np.float64) ** 2).sum()) for r in res.values())
            plan.adjoint(sp, src, rp, plan.residual_scale(rp, res))
        grad = plan.gradient(transform=True)
    else:
        raise ValueError("unknown request kind %r" % req.kind)
    return Result(req.rid, seis, grad, misfit, 0.0, 0.0, 0.0)


def percentiles(latencies: Sequence[float], qs=(50, 99)) -> Dict[str, float]:
    a = np.sort(np.asarray(latencies, np.float64))
    return {"p%d" % q: float(np.percentile(a, q)) if len(a) else float("nan") for q in qs}
