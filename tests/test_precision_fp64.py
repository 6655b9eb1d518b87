"""Errors against an FP64 build of the same scheme.

The oracle's restatement compiled with every float retyped double
(``Oracle(cfg, fp64=True)``, oracle/fdo.h FDO_FP64) is the double-precision
result.  The CUDA path computes in FP32 (FP64 gradient sums) and can store
wave fields in FP16 and saved boundaries in FP16/BF16; each is measured
here against the FP64 build on the same FP32 inputs.

Bars (relative L2, sqrt(sum (d - r)^2 / sum r^2), over all outputs of a case):
  FP32 forward seismograms                      1e-5
  FP16 wave-field storage, forward seismograms  1e-3 energy ratio (the
        reference's FP16 criterion, test_consistency.py), reported as rel L2
  FP16 memory variables (FP32 wave fields)      1e-3
  gradients, FP32 boundaries                    1e-3
  gradients, FP16 / BF16 saved boundaries       1e-3
  serving results (seismograms and gradients)   1e-3
Each test prints its measured errors on lines starting "FP64ERR".
"""
import numpy as np
import pytest

from tests._cases import engine_config, make_case, rel_l2


def _joint_rel(got: dict, ref: dict) -> float:
    num = sum(float(((np.asarray(got[k], np.float64) - ref[k]) ** 2).sum()) for k in ref)
    den = sum(float((np.asarray(ref[k], np.float64) ** 2).sum()) for k in ref)
    assert den > 0
    return float(np.sqrt(num / den))


def _fp64(cfg, model):
    from oracle.oracle import Oracle

    o = Oracle(cfg, fp64=True)
    assert o.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"]) == 0
    return o


# ------------------------------------------------------------------ CPU
@pytest.mark.parametrize("kw", [dict(nd=2, freesurf=1, L=0, nt=200), dict(nd=2, freesurf=0, L=2, src_type=2, nt=200),
                                dict(nd=3, freesurf=1, L=1, nz=28, ny=26, nx=30, nt=80, nab=6)],
                         ids=["2d", "2d_visco", "3d_visco"])
def test_fp64_build_is_the_same_scheme(kw):
    """The FP64 build runs the FP32 build's scheme: its results are float64
    and differ from the FP32 build's only by rounding."""
    from oracle.oracle import Oracle

    cfg, model, acq = make_case(**kw)
    outs = ["vx", "vz", "p"]
    d, g = {}, {}
    for fp64 in (False, True):
        o = Oracle(cfg, fp64=fp64)
        assert o.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"]) == 0
        d[fp64] = o.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
        o.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"],
                  {k: (0.3 * v).astype(np.float32) for k, v in d[fp64].items() if k != "p"})
        g[fp64] = o.gradients()
        o.close()
    assert all(v.dtype == np.float64 for v in d[True].values())
    e_fwd = _joint_rel(d[False], d[True])
    e_grad = max(rel_l2(g[False][k], g[True][k]) for k in ("vp", "vs", "rho"))
    print("FP64ERR oracle-fp32 %s forward %.3g gradient %.3g" % (kw, e_fwd, e_grad))
    assert 0 < e_fwd < 1e-5
    assert 0 < e_grad < 1e-4


# ------------------------------------------------------------------ GPU
@pytest.mark.gpu
@pytest.mark.parametrize("kw", [
    dict(nd=3, freesurf=1, L=2, abs_type=1, src_type=2, nz=64, ny=64, nx=64, nt=400, nab=10, seed=71),
    dict(nd=3, freesurf=1, L=0, abs_type=1, src_type=100, nz=48, ny=44, nx=52, nt=300, nab=8, seed=72),
    dict(nd=2, freesurf=1, L=0, abs_type=1, src_type=100, nz=150, nx=200, nt=1000, nab=20, seed=73),
    dict(nd=2, freesurf=1, L=2, abs_type=1, src_type=100, nz=120, nx=160, nt=800, nab=16, seed=74),
    dict(nd=3, freesurf=0, L=3, abs_type=2, src_type=100, nz=48, ny=40, nx=44, nt=300, nab=8, seed=78),
], ids=["3d_visco_64", "3d_elastic", "2d_psv", "2d_visco", "3d_visco_L3_taper"])
def test_forward_against_fp64(kw, cuda_device):
    import dataclasses

    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(**kw)
    outs = ["vx", "vy", "vz", "p"] if cfg["nd"] == 3 else ["vx", "vz", "p"]
    ref = _fp64(cfg, model).forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
    precs = ("fp32", "fp16") + (("fp16_mem",) if cfg["nd"] == 3 and cfg["L"] > 0 else ())
    for prec in precs:
        plan = Plan(dataclasses.replace(engine_config(cfg), field_precision=prec))
        plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
        got = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
        fam = plan.kernel_family
        plan.close()
        err = _joint_rel(got, ref)
        per = {k: round(rel_l2(got[k], ref[k]), 9) for k in outs}
        print("FP64ERR forward %s %s %s joint %.3g %s" % (kw, prec, fam, err, per))
        if prec == "fp32":
            assert err < 1e-5, err
        elif prec == "fp16_mem":
            assert err < 1e-3, err
        else:
            assert err * err < 1e-3, err


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [
    dict(nd=2, freesurf=1, L=0, abs_type=1, src_type=100, nt=300, seed=75),
    dict(nd=2, freesurf=0, L=0, abs_type=1, src_type=2, nz=80, nx=100, nt=400, nab=14, seed=76),
    dict(nd=3, freesurf=1, L=0, abs_type=1, src_type=100, nz=40, ny=36, nx=44, nt=150, nab=8, seed=77),
], ids=["2d_fs", "2d_force", "3d"])
def test_gradient_against_fp64(kw, cuda_device):
    import dataclasses

    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(**kw)
    outs = ["vx", "vy", "vz"] if cfg["nd"] == 3 else ["vx", "vz"]
    o = _fp64(cfg, model)
    d = o.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
    res = {k: (0.3 * v).astype(np.float32) for k, v in d.items()}
    o.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], res)
    gref = o.gradients()
    got = {}
    for prec in ("fp32", "fp16", "bf16"):
        plan = Plan(dataclasses.replace(engine_config(cfg), precision=prec))
        plan.set_model(model["vp"], model["vs"], model["rho"])
        plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
        plan.zero_gradient()
        plan.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], res)
        g = plan.gradient(transform=True)
        plan.close()
        errs = {k: rel_l2(g[k], gref[k]) for k in ("vp", "vs", "rho")}
        print("FP64ERR gradient %s boundaries %s %s" % (kw, prec, {k: round(v, 9) for k, v in errs.items()}))
        got[prec] = errs
    for prec in ("fp32", "fp16", "bf16"):
        assert max(got[prec].values()) < 1e-3, (prec, got)


@pytest.mark.gpu
def test_serving_results_against_fp64(cuda_device):
    """Requests served concurrently (forward and gradient, 2D and 3D,
    elastic and viscoelastic): every seismogram and gradient within 1e-3 of
    the FP64 build."""
    from seiscl_b200 import serving

    cases = [dict(nd=2, freesurf=1, L=2, nt=300, seed=81), dict(nd=2, freesurf=1, L=0, nt=300, seed=82),
             dict(nd=3, freesurf=1, L=1, nz=32, ny=30, nx=34, nt=120, nab=8, seed=83),
             dict(nd=2, freesurf=0, L=0, nt=300, seed=84, nz=60, nx=70)]
    reqs, refs = [], []
    for i, kw in enumerate(cases):
        cfg, model, acq = make_case(**kw)
        outs = ("vx", "vz")
        kind = "gradient" if i % 2 else "forward"
        o = _fp64(cfg, model)
        d = o.forward(acq["src_pos"], acq["src"], acq["rec_pos"], list(outs), save_boundaries=kind == "gradient")
        obs = None
        gref = None
        if kind == "gradient":
            obs = [{k: (0.7 * v).astype(np.float32) for k, v in d.items()}]
            # the service's adjoint source: residual d - obs, scaled as res_scale
            res = o.residual_scale(acq["rec_pos"], {k: (d[k] - obs[0][k]).astype(np.float32) for k in outs})
            o.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], res)
            gref = o.gradients()
        o.close()
        m = {k: v for k, v in model.items() if v is not None}
        reqs.append(serving.Request(engine_config(cfg), m, [(acq["src_pos"], acq["src"], acq["rec_pos"])], outs,
                                    kind, obs, rid=i))
        refs.append((d, gref))
    with serving.Server(workers=3) as srv:
        res = [f.result(timeout=600) for f in [srv.submit(q) for q in reqs * 2]]
    worst = 0.0
    for i, r in enumerate(res):
        d, gref = refs[i % len(cases)]
        e = _joint_rel(r.seismograms[0], d)
        worst = max(worst, e)
        assert e < 1e-3, (i, e)
        if gref is not None:
            for k in ("vp", "vs", "rho"):
                eg = rel_l2(r.gradient[k], gref[k])
                worst = max(worst, eg)
                assert eg < 1e-3, (i, k, eg)
    print("FP64ERR serving worst %.3g" % worst)
