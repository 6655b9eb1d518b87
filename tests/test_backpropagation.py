"""Backward reconstruction of the forward wave field (the check of the
reference's test_consistency.py:test_backpropagation, which requires the
reconstructed field to vanish inside the absorbing frame to 1e-4).

The adjoint run rebuilds the forward field backwards in time from its final
state, the saved boundary shells and the removed sources; after the last
adjoint step the field is back at the first step's, which is ~0 away from
the source.  Bound here: 3e-3 of the field's peak inside the absorbing
frame (the oracle, with the reference's double-evaluated stencils, stays
below 6e-4; the FP32 engine below 1.2e-3 on these cases).  This exercises
the restated time loop of the oracle
(fdo_driver.c) and of the engine (sfd_capi.cu) as a whole: step order, slice
t-1 injection, source removal after the adjoint update.
"""
import numpy as np
import pytest

from tests._cases import engine_config, make_case

F = 4
RTOL = 3e-3
NAMES = ("vx", "vz", "sxx", "szz", "sxz")
CASES = [dict(nd=2, freesurf=fs, L=0, abs_type=1, src_type=st, nt=400) for fs in (0, 1) for st in (100, 2)]


def _interior(a, cfg):
    nab, NZ, NX = cfg["nab"], cfg["nz"] + 2 * F, cfg["nx"] + 2 * F
    a = a.reshape(NX, NZ)
    z0 = F if cfg["freesurf"] else nab + F
    return a[nab + F:NX - nab - F, z0:NZ - nab - F]


@pytest.mark.parametrize("kw", CASES, ids=lambda k: "fs%d-src%d" % (k["freesurf"], k["src_type"]))
def test_oracle_reconstructs_forward_field(kw):
    from oracle.oracle import Oracle

    cfg, model, acq = make_case(**kw)
    o = Oracle(cfg)
    o.set_model(model["vp"], model["vs"], model["rho"])
    d = o.forward(acq["src_pos"], acq["src"], acq["rec_pos"], ["vx", "vz"], save_boundaries=True)
    peak = {n: np.abs(_interior(o.array("wave", n), cfg)).max() for n in NAMES}
    o.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], {k: 0 * v for k, v in d.items()})
    for n in NAMES:
        assert peak[n] > 0
        assert np.abs(_interior(o.array("wave", n), cfg)).max() < RTOL * peak[n], n


@pytest.mark.gpu
@pytest.mark.parametrize("kw", CASES, ids=lambda k: "fs%d-src%d" % (k["freesurf"], k["src_type"]))
def test_engine_reconstructs_forward_field(kw, cuda_device):
    from seiscl_b200.engine import Plan

    ids = {"vx": 0, "vz": 2, "sxx": 3, "szz": 5, "sxz": 8}
    cfg, model, acq = make_case(**kw)
    plan = Plan(engine_config(cfg))
    plan.set_model(model["vp"], model["vs"], model["rho"])
    d = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], ["vx", "vz"], save_boundaries=True)
    n = plan.nvol
    peak = {k: np.abs(_interior(plan.debug_array(0, ids[k], n), cfg)).max() for k in NAMES}
    plan.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], {k: 0 * v for k, v in d.items()})
    for k in NAMES:
        assert peak[k] > 0
        assert np.abs(_interior(plan.debug_array(0, ids[k], n), cfg)).max() < RTOL * peak[k], k
