"""seiscl_b200.autograd: the adjoint gradient behind torch.autograd against
central finite differences of the forward modelling (GPU).

The check is the gradient test along the gradient direction restricted to
the interior (absorbing layers and the source's neighbourhood excluded):
(L(m + e g) - L(m - e g)) / 2e against <g, g>.  Tolerances are those this
adjoint-state gradient meets on the same cases with the oracle (vp, vs: 10 %;
rho: 40 %): SeisCL's adjoint is not the exact transpose of its discrete
forward scheme.  Measured on a B200 (analytic / central difference):
explosive source vp 1.005, vs 1.065, rho 0.887; vertical force vp 0.973,
vs 1.052, rho 1.337.
"""
import dataclasses

import numpy as np
import pytest

from tests._cases import engine_config, make_case


@pytest.mark.gpu
@pytest.mark.parametrize("src_type", [100, 2])
def test_gradient_matches_central_differences(src_type, cuda_device):
    import torch

    from seiscl_b200.autograd import seismograms
    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(nd=2, freesurf=0, L=0, abs_type=1, src_type=src_type, nt=500, nz=80, nx=90,
                                nab=12)
    plan = Plan(dataclasses.replace(engine_config(cfg), adjoint_reset_psi=True))
    shots = [(acq["src_pos"], acq["src"], acq["rec_pos"])]
    outs = ["vx", "vz"]
    m = {k: torch.tensor(model[k].T.copy(), dtype=torch.float64) for k in ("vp", "vs", "rho")}
    d0 = seismograms(plan, m["vp"], m["vs"], m["rho"], shots, outs).detach().double()
    w = d0 / float((d0 * d0).sum())
    mr = {k: v.clone().requires_grad_(True) for k, v in m.items()}
    (seismograms(plan, mr["vp"], mr["vs"], mr["rho"], shots, outs).double() * w).sum().backward()
    nz, nx, nab = cfg["nz"], cfg["nx"], cfg["nab"]
    zz, xx = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
    xs, zs = acq["src_pos"][0, 0] / cfg["dh"], acq["src_pos"][0, 2] / cfg["dh"]
    mask = torch.tensor(((zz >= nab) & (zz < nz - nab) & (xx >= nab) & (xx < nx - nab)
                         & (np.hypot(xx - xs, zz - zs) > 4)).astype(np.float64))
    tol = {"vp": 0.1, "vs": 0.1, "rho": 0.4}
    for name in ("vp", "vs", "rho"):
        g = mr[name].grad.double() * mask
        assert float(g.abs().max()) > 0, name
        delta = g / g.abs().max()
        eps = 1e-3 * float(m[name].mean())

        def L(sgn):
            a = dict(m)
            a[name] = m[name] + sgn * eps * delta
            return float((seismograms(plan, a["vp"], a["vs"], a["rho"], shots, outs).double() * w).sum())

        fd = (L(1) - L(-1)) / (2 * eps)
        an = float((g * delta).sum())
        print("AUTOGRAD src_type %d %s analytic / central difference %.4f" % (src_type, name, an / fd))
        assert abs(an / fd - 1) < tol[name], (name, an / fd)


@pytest.mark.gpu
def test_checkpointed_plan_behind_autograd(cuda_device):
    """The snapshot-checkpoint recompute strategy behind torch.autograd: the
    same gradient as boundary-saving reconstruction inside the region the
    boundary shells enclose, and the same central-difference check."""
    import torch

    from seiscl_b200.autograd import seismograms
    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(nd=2, freesurf=0, L=0, abs_type=1, src_type=100, nt=400, nz=80, nx=90, nab=12)
    shots = [(acq["src_pos"], acq["src"], acq["rec_pos"])]
    outs = ["vx", "vz"]
    m = {k: torch.tensor(model[k].T.copy(), dtype=torch.float64) for k in ("vp", "vs", "rho")}
    grads = {}
    for K in (0, 25):
        plan = Plan(dataclasses.replace(engine_config(cfg), adjoint_reset_psi=True, checkpoint=K))
        d0 = seismograms(plan, m["vp"], m["vs"], m["rho"], shots, outs).detach().double()
        w = d0 / float((d0 * d0).sum())
        mr = {k: v.clone().requires_grad_(True) for k, v in m.items()}
        (seismograms(plan, mr["vp"], mr["vs"], mr["rho"], shots, outs).double() * w).sum().backward()
        grads[K] = {k: v.grad.double().numpy() for k, v in mr.items()}
        plan.close()
    e = cfg["nab"] + 6
    for name in ("vp", "vs", "rho"):
        a, b = grads[25][name][e:-e, e:-e], grads[0][name][e:-e, e:-e]
        assert np.abs(b).max() > 0, name
        assert np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()) < 2e-4, name


def test_force_sources_need_reset_psi():
    """seismograms() refuses force sources on a plan that carries the forward
    CPML memory into the adjoint (their gradient would be dominated by it);
    the check runs before any device work."""
    import types

    import torch

    from seiscl_b200.autograd import seismograms

    plan = types.SimpleNamespace(cfg=types.SimpleNamespace(adjoint_reset_psi=False))
    m = torch.ones((8, 8))
    rp = np.zeros((1, 8), np.float32)
    src = np.zeros((1, 10), np.float32)
    for ty in (0, 1, 2):
        sp = np.array([[10.0, 0.0, 10.0, 0, ty]], np.float32)
        with pytest.raises(ValueError):
            seismograms(plan, m, m, m, [(sp, src, rp)], ["vx"])
