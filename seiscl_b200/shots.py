"""Shot-parallel execution over ranks (one process per GPU).

Shots are independent, so they are split over the ranks of a
``torch.distributed`` process group with no data-path collective; the
per-shot results are combined once at the end with one sum-reduction per
output, as the reference combines its MPI groups (src/time_stepping.c:705-722
for the split, src/Out_MPI.c:70-160 for the reductions of seismograms,
residuals, misfit and gradients).  With NCCL the reductions run on the GPU
over NVLink/NVSwitch; with gloo (tests, CPU) on the host.
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
