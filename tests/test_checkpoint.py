"""Checkpointed gradients (``Config.checkpoint = K``).

The forward run keeps a snapshot of its whole state every K steps; the
adjoint recomputes each K-step segment from its snapshot and reads the
forward field it needs instead of reconstructing it by backpropagation and
boundary injection (the reference's BACK_PROP_TYPE 1,
src/time_stepping.c:862-940).  Inside the region the saved boundary shells
enclose, backpropagation reconstructs the forward field exactly up to
rounding, so there both gradients agree; in the absorbing layers the
reconstruction is not the forward field and the two differ.  For
viscoelastic media, where backpropagation is unstable (the reference flags
it, src/update_adjs2D.cl:232), the checkpointed gradient stays close to the
elastic one as attenuation vanishes.
"""
import dataclasses

import numpy as np
import pytest

from tests._cases import engine_config, make_case, rel_l2


def _interior(a, cfg, top):
    m = cfg["nab"] + cfg["fdorder"] // 2 + 2
    if cfg["nd"] == 3:
        return a[m:-m, m:-m, top:-m]
    return a[m:-m, top:-m]


def _gradient(cfg, model, acq, outs, **extra):
    from seiscl_b200.engine import Plan

    plan = Plan(dataclasses.replace(engine_config(cfg), **extra))
    plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    plan.zero_gradient()
    d = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
    plan.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], {k: (0.3 * v).astype(np.float32) for k, v in d.items()})
    g = plan.gradient(transform=False)
    nbytes = plan.device_bytes
    plan.close()
    return d, g, nbytes


CASES = [
    (dict(nd=2, freesurf=0, L=0, abs_type=1, src_type=100, nt=200, seed=111), 50),
    (dict(nd=2, freesurf=0, L=0, abs_type=1, src_type=2, nt=200, seed=112, fdorder=4), 7),
    (dict(nd=2, freesurf=1, L=0, abs_type=1, src_type=100, nt=200, seed=113), 1),
    (dict(nd=2, freesurf=0, L=0, abs_type=2, src_type=100, nt=200, seed=114), 300),
    (dict(nd=3, freesurf=0, L=0, abs_type=1, src_type=100, nz=36, ny=32, nx=36, nt=100, nab=8, seed=115), 25),
    (dict(nd=3, freesurf=1, L=0, abs_type=1, src_type=2, nz=38, ny=30, nx=34, nt=100, nab=8, seed=116), 30),
]


@pytest.mark.gpu
@pytest.mark.parametrize("kw,K", CASES, ids=["2d_K50", "2d_o4_K7", "2d_fs_K1", "2d_taper_Knt", "3d_vector_K25",
                                             "3d_general_fs_K30"])
def test_checkpointed_gradient_matches_backpropagation_inside(kw, K, cuda_device):
    cfg, model, acq = make_case(**kw)
    outs = ["vx", "vy", "vz"] if cfg["nd"] == 3 else ["vx", "vz"]
    d1, g1, _ = _gradient(cfg, model, acq, outs)
    d2, g2, _ = _gradient(cfg, model, acq, outs, checkpoint=K)
    for k in outs:   # the forward runs are the same
        assert np.array_equal(d1[k], d2[k]), k
    top = 2 * (cfg["fdorder"] // 2) + 4 if cfg["freesurf"] else cfg["nab"] + cfg["fdorder"] // 2 + 2
    for k in ("M", "mu", "rho"):
        a, b = _interior(g2[k], cfg, top), _interior(g1[k], cfg, top)
        assert np.abs(b).max() > 0, k
        assert rel_l2(a, b) < 2e-4, (k, rel_l2(a, b))


@pytest.mark.gpu
def test_checkpointed_viscoelastic_gradient_is_stable(cuda_device):
    """With weak attenuation the viscoelastic gradient must approach the
    elastic one: the checkpointed one does (correlation 0.99999 and more for
    M, mu and rho), the backpropagated one, reproduced from the reference,
    does not (0.996, 0.19 and 0.29 on this case)."""
    cfg, model, acq = make_case(nd=2, freesurf=0, L=1, abs_type=1, src_type=100, nt=300, seed=117)
    weak = dict(model, taup=np.full_like(model["taup"], 0.01), taus=np.full_like(model["taus"], 0.01))
    el_cfg = dict(cfg, L=0)
    el = dict(model, taup=None, taus=None)
    _, ge, _ = _gradient(el_cfg, el, acq, ["vx", "vz"])
    _, gc, _ = _gradient(cfg, weak, acq, ["vx", "vz"], checkpoint=40)
    _, gb, _ = _gradient(cfg, weak, acq, ["vx", "vz"])
    top = cfg["nab"] + 6

    def corr(a, b):
        a = _interior(a, cfg, top).ravel().astype(np.float64)
        b = _interior(b, cfg, top).ravel().astype(np.float64)
        a /= np.abs(a).max()
        b /= np.abs(b).max()
        return float(np.dot(a, b) / np.sqrt(np.dot(a, a) * np.dot(b, b)))

    for k in ("M", "mu", "rho"):
        cc = corr(gc[k], ge[k])
        cb = corr(gb[k], ge[k]) if np.isfinite(gb[k]).all() else float("nan")
        print("%s: checkpointed %.6f backpropagated %s" % (k, cc, cb))
        assert np.isfinite(cc) and cc > 0.999, (k, cc)
    assert all(np.isfinite(v).all() for v in gc.values() if v is not None)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp16", "bf16"])
def test_checkpoint_stores_in_half_precision(prec, cuda_device):
    """Snapshots and segment stores in FP16 (power-of-two scaled) or BF16:
    the gradient stays within 1e-3 of the FP32-store one, and the plan holds
    what ``sfd_footprint`` says."""
    from seiscl_b200 import engine

    cfg, model, acq = make_case(nd=2, freesurf=1, L=0, abs_type=1, src_type=100, nt=200, seed=118)
    _, g32, _ = _gradient(cfg, model, acq, ["vx", "vz"], checkpoint=20)
    _, gh, nbytes = _gradient(cfg, model, acq, ["vx", "vz"], checkpoint=20, precision=prec)
    for k in ("M", "mu", "rho"):
        assert rel_l2(gh[k], g32[k]) < 1e-3, (k, rel_l2(gh[k], g32[k]))
    ec = dataclasses.replace(engine_config(cfg), checkpoint=20, precision=prec)
    assert nbytes == engine.footprint(ec, True, 1, 2 * len(acq["rec_pos"]))


FP16_FIELD_CASES = [
    (dict(nd=2, freesurf=1, L=0, abs_type=1, src_type=100, nt=200, seed=119), 25, "fp32"),
    (dict(nd=2, freesurf=0, L=2, abs_type=1, src_type=100, nt=200, seed=120), 40, "fp16"),
    (dict(nd=3, freesurf=1, L=0, abs_type=1, src_type=100, nz=36, ny=32, nx=36, nt=100, nab=8, seed=121), 25, "fp32"),
    (dict(nd=3, freesurf=0, L=2, abs_type=1, src_type=2, nz=36, ny=32, nx=36, nt=100, nab=8, seed=122), 20, "bf16"),
]
# relative L2 of the gradient with FP16 wave fields against FP32 wave fields
# (same checkpointing): the rounding of the stored fields carried through the
# residuals and the correlation; measured on a B200 1.7e-4 - 5.5e-3
FP16_FIELD_GRAD_TOL = 1e-2


@pytest.mark.gpu
@pytest.mark.parametrize("kw,K,prec", FP16_FIELD_CASES,
                         ids=["2d_fs", "2d_visco_fp16store", "3d_fs", "3d_visco_bf16store"])
def test_fp16_wave_fields_in_checkpointed_gradient(kw, K, prec, cuda_device):
    """FP16 wave-field storage in the forward and recomputed runs of a
    checkpointed gradient (the adjoint fields stay FP32 and read unscaled
    parameters): the forward seismograms are those of an FP16 modelling run,
    bit for bit; the gradient is within FP16_FIELD_GRAD_TOL of the one with
    FP32 wave fields; the plan holds what ``sfd_footprint`` says."""
    from seiscl_b200 import engine

    cfg, model, acq = make_case(**kw)
    outs = ["vx", "vy", "vz"] if cfg["nd"] == 3 else ["vx", "vz"]
    _, g32, _ = _gradient(cfg, model, acq, outs, checkpoint=K, precision=prec)
    dh, gh, nbytes = _gradient(cfg, model, acq, outs, checkpoint=K, precision=prec, field_precision="fp16")
    plan = engine.Plan(dataclasses.replace(engine_config(cfg), field_precision="fp16"))
    plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    dm = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
    plan.close()
    for k in outs:
        assert np.array_equal(dh[k], dm[k]), k
    errs = {k: rel_l2(gh[k], g32[k]) for k in ("M", "mu", "rho")}
    print("FP16 wave fields, checkpointed gradient vs FP32 fields:", errs)
    for k, e in errs.items():
        assert np.abs(g32[k]).max() > 0 and np.isfinite(gh[k]).all(), k
        assert e < FP16_FIELD_GRAD_TOL, (k, e)
    ec = dataclasses.replace(engine_config(cfg), checkpoint=K, precision=prec, field_precision="fp16")
    assert nbytes == engine.footprint(ec, True, 1, len(outs) * len(acq["rec_pos"]))


def test_checkpoint_configuration_checks():
    from seiscl_b200 import engine

    ok = engine.Config(N=[40, 50], ND=2, NT=100, nab=8, checkpoint=10)
    f0 = engine.footprint(dataclasses.replace(ok, checkpoint=0), True, 1, 20)
    f1 = engine.footprint(ok, True, 1, 20)
    f2 = engine.footprint(dataclasses.replace(ok, checkpoint=50), True, 1, 20)
    assert len({f0, f1, f2}) == 3
    # FP16 wave fields: snapshots of half the bytes, plus the adjoint's unscaled parameters
    fh = engine.footprint(dataclasses.replace(ok, field_precision="fp16"), True, 1, 20)
    assert fh < f1
    for bad in (dict(checkpoint=-1), dict(checkpoint=5, back_prop_type=2), dict(checkpoint=5, ND=22, N=[40, 50]),
                dict(checkpoint=5, batch=2), dict(checkpoint=5, field_precision="fp16", hout=1)):
        with pytest.raises(engine.SeisCLEngineError):
            engine.footprint(dataclasses.replace(ok, **bad), True, 1, 20)
