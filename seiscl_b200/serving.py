"""Modelling service: a queue of forward / gradient requests served by a pool
of workers sharing one GPU.

Each worker thread owns its plans (one per distinct grid configuration, kept
in a small LRU cache) and therefore its own CUDA streams; requests are taken
from one FIFO queue as soon as a worker is free (continuous batching at
request granularity), so small grids from different requests run
concurrently on the GPU while a large one occupies a single worker.  A
request's result depends only on the request: every shot starts from zeroed
wave fields on a plan whose model is set from the request, so the output is
the same whatever else is in flight (tested).

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


class Server:
    """``Server(workers=4)``; ``submit(request) -> Future[Result]``;
    ``close()`` drains the queue and stops the workers."""

    def __init__(self, workers: int = 4, plans_per_worker: int = 4, device: Optional[int] = None):
        self._q: "queue.Queue" = queue.Queue()
        self._closed = False
        self._device = device
        self._plans_per_worker = plans_per_worker
        self._threads = [threading.Thread(target=self._run, name="sfd-worker-%d" % i, daemon=True)
                         for i in range(workers)]
        for t in self._threads:
            t.start()

    def submit(self, req: Request) -> Future:
        if self._closed:
            raise RuntimeError("server closed")
        fut: Future = Future()
        self._q.put((req, fut, time.perf_counter()))
        return fut

    def close(self):
        self._closed = True
        for _ in self._threads:
            self._q.put(None)
        for t in self._threads:
            t.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------ worker
    def _run(self):
        if self._device is not None:
            import torch

            torch.cuda.set_device(self._device)
        plans: "collections.OrderedDict" = collections.OrderedDict()
        try:
            while True:
                item = self._q.get()
                if item is None:
                    return
                req, fut, t_submit = item
                if not fut.set_running_or_notify_cancel():
                    continue
                t_start = time.perf_counter()
                try:
                    plan = self._plan(plans, req.config)
                    res = serve(plan, req)
                    res.t_submit, res.t_start, res.t_done = t_submit, t_start, time.perf_counter()
                    fut.set_result(res)
                except BaseException as exc:  # reported through the future
                    fut.set_exception(exc)
        finally:
            for p in plans.values():
                p.close()

    def _plan(self, plans, cfg):
        k = _key(cfg)
        if k in plans:
            plans.move_to_end(k)
            return plans[k]
        if len(plans) >= self._plans_per_worker:
            _, old = plans.popitem(last=False)
            old.close()
        plans[k] = engine.Plan(cfg)
        return plans[k]


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
