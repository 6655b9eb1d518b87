"""CUDA path vs the CPU oracle at the benchmarked configurations.

The other parity tests run small grids; these run the default kernels on
the grids, boundaries and acquisitions the benchmark numbers are quoted on:

* psv2d: 2D P-SV elastic forward, 300 x 400, NT 2000, 8th order, 20-cell
  CPML, free surface, explosive source at (z=5, x=200), 200 receivers at
  z=5 every 2 cells recording vx and vz -- the full shot;
* visco3d: the 3D viscoelastic grid of the headline number (256^3, L=2,
  8th order, 20-cell CPML with the whole-quad z-slab path, free surface,
  six layers, vertical force at the centre top, 64 x 64 receivers at
  4-cell spacing recording vx, vy, vz) for 100 time steps (the oracle
  advances ~1e8 cell-updates per second on the host cores);
* fwi2d: the 2D FWI gradient shape (300 x 1000, 4th order, vs = 0, 500
  receivers, explosive source) for 600 time steps: forward with saved
  boundaries, adjoint, gradient.

Each is also compared with the oracle's FP64 build (the same scheme with
every float retyped double) for the error table.  Tolerances are those of
the small-grid parity tests: 2e-5 relative L2 for seismograms, 2e-4 for
gradients; FP64 comparisons 1e-5.  Set SEISCL_PARITY_REPORT to a file path
to have the measured errors appended to it as JSON lines.
"""
import json
import os

import numpy as np
import pytest

from tests._cases import rel_l2

FWD_TOL = 2e-5
GRAD_TOL = 2e-4
FP64_TOL = 1e-5


def _report(**kw):
    path = os.environ.get("SEISCL_PARITY_REPORT")
    if path:
        with open(path, "a") as fh:
            fh.write(json.dumps(kw) + "\n")


def _shifted_ricker(f0, nt, dt, t0):
    t = np.arange(nt) * dt - t0
    a = (np.pi * f0 * t) ** 2
    return ((1.0 - 2.0 * a) * np.exp(-a)).astype(np.float32)[None, :]


def _forward_pair(name, nt=None, src=None):
    import bench
    from oracle.oracle import Oracle
    from seiscl_b200.engine import Plan

    w, model, acq = bench.build_workload(name)
    if nt is not None:
        w["nt"] = nt
    src = acq["src"][:, :w["nt"]] if src is None else src
    cfg = bench.oracle_config(w)
    plan = Plan(bench.engine_config(w))
    plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    assert plan.kernel_family in ("2d", "vector")
    d_gpu = plan.forward(acq["src_pos"], src, acq["rec_pos"], acq["outputs"])
    del plan
    out = {}
    for fp64 in (False, True):
        ora = Oracle(cfg, fp64=fp64)
        assert ora.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"]) == 0
        out[fp64] = ora.forward(acq["src_pos"], src, acq["rec_pos"], acq["outputs"])
        ora.close()
    return d_gpu, out[False], out[True]


def _check_forward(tag, d_gpu, d_ref, d_64):
    for name in d_ref:
        assert np.abs(d_ref[name]).max() > 0, name
        e32 = rel_l2(d_gpu[name], d_ref[name])
        e64 = rel_l2(d_gpu[name], d_64[name])
        eo = rel_l2(d_ref[name], d_64[name])
        _report(case=tag, output=name, gpu_vs_oracle=e32, gpu_vs_fp64=e64, oracle_vs_fp64=eo)
        assert e32 < FWD_TOL, (name, e32)
        assert e64 < FP64_TOL, (name, e64)


@pytest.mark.gpu
def test_psv2d_full_shot_matches_oracle(cuda_device):
    d_gpu, d_ref, d_64 = _forward_pair("psv2d")
    _check_forward("psv2d 300x400 NT2000", d_gpu, d_ref, d_64)


@pytest.mark.gpu
def test_visco3d_256_matches_oracle(cuda_device):
    # 100 steps of the headline grid; the source peaks at 60 ms so the
    # wave field is well developed within them
    d_gpu, d_ref, d_64 = _forward_pair("visco3d", nt=100, src=_shifted_ricker(10.0, 100, 1e-3, 0.06))
    _check_forward("visco3d 256^3 NT100", d_gpu, d_ref, d_64)


@pytest.mark.gpu
def test_fwi2d_gradient_shape_matches_oracle(cuda_device):
    import bench
    from oracle.oracle import Oracle
    from seiscl_b200.engine import Plan

    w, true, start, shots = bench.build_gradient_workload("fwi2d", 1)
    nt = 600
    w["nt"] = nt
    sp, src, rp = shots[0]
    src = _shifted_ricker(w["src_f"], nt, w["dt"], 0.15)
    outs = w["outputs"]
    cfg = bench.oracle_config(w)
    ora = Oracle(cfg)
    assert ora.set_model(start["vp"], start["vs"], start["rho"]) == 0
    d_ref = ora.forward(sp, src, rp, outs, save_boundaries=True)
    res = {k: (0.3 * v).astype(np.float32) for k, v in d_ref.items()}
    ora.clear_gradients()
    ora.adjoint(sp, src, rp, res)
    g_ref = ora.gradients()

    ec = bench.engine_config(w)
    plan = Plan(ec)
    plan.set_model(start["vp"], start["vs"], start["rho"])
    d_gpu = plan.forward(sp, src, rp, outs, save_boundaries=True)
    for k in d_ref:
        e = rel_l2(d_gpu[k], d_ref[k])
        _report(case="fwi2d 300x1000 NT600 forward", output=k, gpu_vs_oracle=e)
        assert e < FWD_TOL, (k, e)
    plan.zero_gradient()
    plan.adjoint(sp, src, rp, res)
    g = plan.gradient(transform=False)
    # vs = 0: the mu gradient is not defined (1/mu^2 in the reference's
    # adjoint stress kernel); M and rho are the acoustic gradients
    for ours, theirs in (("M", "rawM"), ("rho", "rawrho")):
        assert np.abs(g_ref[theirs]).max() > 0, theirs
        e = rel_l2(g[ours], g_ref[theirs])
        _report(case="fwi2d 300x1000 NT600 gradient", output=ours, gpu_vs_oracle=e)
        assert e < GRAD_TOL, (ours, e)
