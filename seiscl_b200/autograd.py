"""torch.autograd binding: material parameters -> seismograms.

``seismograms(plan, vp, vs, rho, shots, outputs)`` runs the forward
modelling of every shot on the plan's GPU and returns a tensor
``[nshot][nout][nrec][NT]``.  Its backward pass is the reference's
boundary-saving adjoint (src/time_stepping.c:862-940): the incoming
gradient of each seismogram is the adjoint source, scaled by ``res_scale``
(src/residuals.c:452-568) exactly as SeisCL scales its L2 residuals, and the
accumulated kernels go through ``transf_grad`` (src/calc_grad.c:975-1107) to
the (vp, vs, rho) parametrisation.  For an L2 misfit this is SeisCL's own
gradient; for any other loss it is the same adjoint driven by dL/dd.

The backward pass re-runs the forward modelling of each shot with boundary
saving before its adjoint (one plan holds the boundaries of one shot), so a
backward costs one forward plus one adjoint per shot.  The gradient is zeroed
in the absorbing layers (the top one only without a free surface), where the
backward reconstruction of the forward field does not hold, as SeisCL's
``read_grad(cropgrad=True)`` does (SeisCL.py:595-601).

Accuracy: this is an adjoint-state gradient of the continuous equations
evaluated on the grid, not the exact adjoint of the discrete scheme.  Checked
against central finite differences along the gradient direction (interior,
no free surface) it agrees to a few percent for vp and vs and to tens of
percent for rho; near a free surface it is less accurate.  Force sources
(types 0, 1, 2) need a plan created with ``adjoint_reset_psi=True``, and
``seismograms`` refuses them otherwise: the reference's adjoint carries the
forward CPML memory over, which then dominates the adjoint field and makes
the gradient wrong by orders of magnitude.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np
import torch

from .engine import Plan


def _host(t: torch.Tensor) -> np.ndarray:
    """A model tensor [NZ, (NY,) NX] (SeisCL orientation) in the engine's host
    layout [nx][(ny)][nz], z fastest."""
    return np.ascontiguousarray(t.detach().to("cpu", torch.float32).numpy().T)


class _Seismograms(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vp, vs, rho, plan: Plan, shots, outputs):
        ctx.plan, ctx.shots, ctx.outputs = plan, shots, list(outputs)
        ctx.save_for_backward(vp, vs, rho)
        plan.set_model(_host(vp), _host(vs), _host(rho))
        out = []
        for sp, src, rp in shots:
            d = plan.forward(sp, src, rp, ctx.outputs)
            out.append(np.stack([d[k] for k in ctx.outputs]))
        return torch.from_numpy(np.stack(out)).to(vp.device)

    @staticmethod
    def backward(ctx, grad_out):
        vp, vs, rho = ctx.saved_tensors
        plan = ctx.plan
        plan.set_model(_host(vp), _host(vs), _host(rho))
        plan.zero_gradient()
        go = grad_out.detach().to("cpu", torch.float32).numpy()
        for i, (sp, src, rp) in enumerate(ctx.shots):
            plan.forward(sp, src, rp, [], save_boundaries=True)
            res = {k: np.ascontiguousarray(go[i, j]) for j, k in enumerate(ctx.outputs)}
            plan.adjoint(sp, src, rp, plan.residual_scale(rp, res))
        g = plan.gradient(transform=True)
        nab = int(plan.cfg.nab)
        for a in g.values():            # host layout [nx][(ny)][nz]
            a[:nab] = 0
            a[-nab:] = 0
            if a.ndim == 3:
                a[:, :nab] = 0
                a[:, -nab:] = 0
            a[..., -nab:] = 0
            if not plan.cfg.freesurf:
                a[..., :nab] = 0
        names = {0: ("vp", "vs"), 1: ("M", "mu"), 2: ("Ip", "Is")}[plan.cfg.param_type]
        to_t = lambda a, like: torch.from_numpy(np.ascontiguousarray(a.T)).to(like.device, like.dtype)
        return to_t(g[names[0]], vp), to_t(g[names[1]], vs), to_t(g["rho"], rho), None, None, None


def seismograms(plan: Plan, vp: torch.Tensor, vs: torch.Tensor, rho: torch.Tensor, shots: Sequence,
                outputs: Sequence[str]) -> torch.Tensor:
    """Differentiable forward modelling.

    ``vp``, ``vs``, ``rho``: N-shaped tensors ([NZ, NX] or [NZ, NY, NX]);
    ``shots``: sequence of (src_pos [nsrc][5], src [nsrc][NT], rec_pos
    [nrec][8]) host arrays; ``outputs``: seismogram names ("vx", "vz", "p",
    ...).  Returns [nshot][len(outputs)][nrec][NT] on vp's device; every shot
    must have the same receiver count.  Raises ValueError for force sources
    on a plan without ``adjoint_reset_psi`` (see the module docstring)."""
    shots = list(shots)
    if not plan.cfg.adjoint_reset_psi:
        for sp, _, _ in shots:
            types = np.asarray(sp, np.float32).reshape(-1, 5)[:, 4].astype(int)
            if np.isin(types, (0, 1, 2)).any():
                raise ValueError("force sources need a plan created with adjoint_reset_psi=True: with the "
                                 "forward run's CPML memory carried into the adjoint (the reference's "
                                 "behaviour) their gradient is dominated by it")
    return _Seismograms.apply(vp, vs, rho, plan, shots, tuple(outputs))
