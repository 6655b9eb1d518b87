"""Shot-parallel execution over ranks (one process per GPU).

Shots are independent, so they are split over the ranks of a
``torch.distributed`` process group with no data-path collective; the
per-shot results are combined once at the end, as the reference combines
its MPI groups (src/time_stepping.c:705-722 for the split,
src/Out_MPI.c:70-160 for the outputs): the traces (and movie frames) each
rank computed are gathered -- one all-gather of each rank's block of rows,
in the arrays' own type -- and the misfit and gradients, which every shot
adds to, are summed in FP64.  With NCCL the collectives run on the GPU over
NVLink/NVSwitch; with gloo (tests, CPU) on the host.
"""
from __future__ import annotations

from typing import Dict, Optional, Tuple

import numpy as np


def shot_range(ns: int, rank: int, world: int) -> Tuple[int, int]:
    """[smin, smax) of the shots processed by group ``rank`` of ``world``.

    Contiguous blocks; the first ``ns % world`` groups take one shot more
    (src/time_stepping.c:705-722)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank %d outside a group of %d" % (rank, world))
    base, extra = divmod(int(ns), int(world))
    smin = rank * base + min(rank, extra)
    return smin, smin + base + (1 if rank < extra else 0)


def dist_context():
    """(rank, world, group-is-NCCL) of the default process group, or
    (0, 1, False) when torch.distributed is not initialised."""
    try:
        import torch.distributed as dist
    except Exception:  # torch without distributed support
        return 0, 1, False
    if not (dist.is_available() and dist.is_initialized()):
        return 0, 1, False
    return dist.get_rank(), dist.get_world_size(), dist.get_backend() == "nccl"


def gather_rows(arrays: Dict[str, np.ndarray], lo: int, hi: int, device: Optional[str] = None) -> Dict[str, np.ndarray]:
    """Every array with rows [lo, hi) (axis 0) taken from the rank that owns
    them: each rank passes its own [lo, hi), the blocks of all ranks must
    tile the rows, and every rank passes the same keys, shapes and dtypes
    (float32 here).  One all-gather of one padded buffer per rank; the
    values arrive unchanged (no arithmetic)."""
    import torch
    import torch.distributed as dist

    rank, world, nccl = dist_context()
    if world == 1:
        return {k: np.array(v, copy=True) for k, v in arrays.items()}
    keys = list(arrays)
    dev = device or ("cuda" if nccl else "cpu")
    bounds = torch.tensor([lo, hi], dtype=torch.int64, device=dev)
    allb = [torch.zeros_like(bounds) for _ in range(world)]
    dist.all_gather(allb, bounds)
    allb = [tuple(int(x) for x in b.cpu()) for b in allb]
    maxrows = max(h - l for l, h in allb)
    widths = [int(np.prod(np.asarray(arrays[k]).shape[1:])) for k in keys]
    row = sum(widths)
    mine = np.zeros((maxrows, row), np.float32)
    o = 0
    for k, wd in zip(keys, widths):
        a = np.asarray(arrays[k], np.float32).reshape(len(arrays[k]), -1)
        mine[:hi - lo, o:o + wd] = a[lo:hi]
        o += wd
    t = torch.from_numpy(mine).to(dev)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    out = {k: np.array(arrays[k], copy=True) for k in keys}
    for (l, h), part in zip(allb, parts):
        blk = part.cpu().numpy()[:h - l]
        o = 0
        for k, wd in zip(keys, widths):
            out[k][l:h] = blk[:, o:o + wd].reshape((h - l,) + np.asarray(arrays[k]).shape[1:])
            o += wd
    return out


def allreduce_sum(arrays: Dict[str, np.ndarray], device: Optional[str] = None) -> Dict[str, np.ndarray]:
    """Element-wise sum of every array over all ranks, in FP64, returned in
    each input's dtype.  Every rank must pass the same keys, shapes and
    order.  One flat buffer, so one collective, whatever the number of
    arrays."""
    import torch
    import torch.distributed as dist

    rank, world, nccl = dist_context()
    if world == 1:
        return {k: np.array(v, copy=True) for k, v in arrays.items()}
    keys = list(arrays)
    flat = np.concatenate([np.asarray(arrays[k], np.float64).ravel() for k in keys]) if keys else np.zeros(0)
    dev = device or ("cuda" if nccl else "cpu")
    t = torch.from_numpy(flat).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    flat = t.cpu().numpy()
    out, o = {}, 0
    for k in keys:
        a = np.asarray(arrays[k])
        out[k] = flat[o:o + a.size].reshape(a.shape).astype(a.dtype)
        o += a.size
    return out
