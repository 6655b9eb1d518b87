"""CUDA path vs the CPU oracle on the same seeded inputs.

Forward seismograms and adjoint gradients go through the C ABI
(libseiscl_b200.so).  The oracle is the C restatement in oracle/ (pinned
bit-exact to the reference kernels by tests/test_oracle_pin.py).

Tolerances (relative L2 over each output):
  forward seismograms   2e-5   (FP32 with FMA vs the reference's
                                 double-accumulated stencils)
  raw gradients         2e-4   (FP64 accumulation here, FP32 in the reference)
"""
import numpy as np
import pytest

from tests._cases import engine_config, make_case, rel_l2

FWD_TOL = 2e-5
# TMA kernels vs general kernels: same operation order except that the TMA
# kernels multiply by FP32 reciprocals of dt, 1 + eta/2 and the CPML K where
# the general kernels divide (a last-bit difference per coefficient)
FAST_TOL = 5e-6
GRAD_TOL = 2e-4

FORWARD_CASES = [
    dict(nd=2, freesurf=1, L=0, abs_type=1, src_type=100),
    dict(nd=2, freesurf=0, L=1, abs_type=1, src_type=2),
    dict(nd=2, freesurf=1, L=2, abs_type=1, src_type=100),
    dict(nd=2, freesurf=0, L=0, abs_type=2, src_type=0),
    dict(nd=2, freesurf=1, L=0, abs_type=1, src_type=100, fdorder=4),
    dict(nd=2, freesurf=0, L=0, abs_type=1, src_type=100, fdorder=12, nz=50, nx=46),
    dict(nd=3, freesurf=1, L=0, abs_type=1, src_type=100, nz=36, ny=34, nx=38, nt=120, nab=8),
    dict(nd=3, freesurf=1, L=2, abs_type=1, src_type=2, nz=36, ny=34, nx=38, nt=120, nab=8),
    dict(nd=3, freesurf=0, L=1, abs_type=2, src_type=1, nz=36, ny=34, nx=38, nt=120, nab=8),
]


def _outputs(nd):
    return ["vx", "vy", "vz", "p"] if nd == 3 else ["vx", "vz", "p"]


def _run_pair(kw, grad=False):
    from oracle.oracle import Oracle
    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(**kw)
    outs = _outputs(cfg["nd"])
    ora = Oracle(cfg)
    assert ora.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"]) == 0
    d_ref = ora.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=grad)
    plan = Plan(engine_config(cfg))
    plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    d_gpu = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=grad)
    return cfg, model, acq, ora, plan, d_ref, d_gpu


@pytest.mark.gpu
@pytest.mark.parametrize("kw", FORWARD_CASES, ids=lambda k: "-".join("%s%s" % (a, b) for a, b in k.items()))
def test_forward_matches_oracle(kw, cuda_device):
    cfg, model, acq, ora, plan, d_ref, d_gpu = _run_pair(kw)
    for name in d_ref:
        ref = d_ref[name]
        assert np.abs(ref).max() > 0, name
        err = rel_l2(d_gpu[name], ref)
        assert err < FWD_TOL, (name, err)


GRAD_CASES = [
    dict(nd=2, freesurf=1, L=0, abs_type=1, src_type=100),
    dict(nd=2, freesurf=0, L=0, abs_type=1, src_type=2),
    dict(nd=2, freesurf=0, L=0, abs_type=2, src_type=100),
    dict(nd=3, freesurf=1, L=0, abs_type=1, src_type=100, nz=36, ny=34, nx=38, nt=100, nab=8),
]


@pytest.mark.gpu
@pytest.mark.parametrize("kw", GRAD_CASES, ids=lambda k: "-".join("%s%s" % (a, b) for a, b in k.items()))
def test_gradient_matches_oracle(kw, cuda_device):
    cfg, model, acq, ora, plan, d_ref, d_gpu = _run_pair(kw, grad=True)
    # residuals: a fixed fraction of the recorded data, as adjoint sources
    res = {k: (0.3 * v).astype(np.float32) for k, v in d_ref.items() if k != "p"}
    ora.clear_gradients()
    ora.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], res)
    g_ref = ora.gradients()
    plan.zero_gradient()
    plan.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], res)
    g_raw = plan.gradient(transform=False)
    for ours, theirs in (("M", "rawM"), ("mu", "rawmu"), ("rho", "rawrho")):
        assert np.abs(g_ref[theirs]).max() > 0, theirs
        err = rel_l2(g_raw[ours], g_ref[theirs])
        assert err < GRAD_TOL, (ours, err)
    g_t = plan.gradient(transform=True)
    for name in ("vp", "vs", "rho"):
        err = rel_l2(g_t[name], g_ref[name])
        assert err < GRAD_TOL, (name, err)


@pytest.mark.gpu
def test_gradient_accumulates_over_shots(cuda_device):
    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(nd=2, nt=120)
    plan = Plan(engine_config(cfg))
    plan.set_model(model["vp"], model["vs"], model["rho"])
    d = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], ["vx", "vz"], save_boundaries=True)
    plan.zero_gradient()
    plan.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], d)
    g1 = plan.gradient(transform=False)
    plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], ["vx", "vz"], save_boundaries=True)
    plan.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], d)
    g2 = plan.gradient(transform=False)
    for k in g1:
        assert rel_l2(g2[k], 2 * g1[k]) < 1e-6


@pytest.mark.gpu
def test_adjoint_requires_forward(cuda_device):
    from seiscl_b200.engine import Plan, SeisCLEngineError

    cfg, model, acq = make_case(nd=2, nt=20)
    plan = Plan(engine_config(cfg))
    plan.set_model(model["vp"], model["vs"], model["rho"])
    with pytest.raises(SeisCLEngineError) as e:
        plan.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], {"vx": np.zeros((len(acq["rec_pos"]), 20))})
    assert e.value.code == -5


FAST_CASES = [
    # TMA-eligible (8th order, nz % 4 == 0): ragged y/x tiles, several x chunks
    dict(nd=3, freesurf=1, L=2, abs_type=1, src_type=100, nz=36, ny=29, nx=31, nt=80, nab=6),
    dict(nd=3, freesurf=0, L=0, abs_type=1, src_type=2, nz=68, ny=35, nx=22, nt=60, nab=5),
    dict(nd=3, freesurf=0, L=1, abs_type=2, src_type=0, nz=40, ny=20, nx=44, nt=60, nab=6),
    dict(nd=3, freesurf=1, L=3, abs_type=1, src_type=100, nz=36, ny=18, nx=40, nt=60, nab=6),
    # nab % 4 == 0: the vectorised kernels' whole-quad z-slab CPML path; the
    # last case is below nz = 2 nab + 4, which takes the per-cell path
    dict(nd=3, freesurf=0, L=2, abs_type=1, src_type=100, nz=40, ny=30, nx=34, nt=60, nab=8),
    dict(nd=3, freesurf=1, L=1, abs_type=1, src_type=2, nz=44, ny=26, nx=30, nt=60, nab=4),
    dict(nd=3, freesurf=1, L=0, abs_type=1, src_type=1, nz=16, ny=26, nx=22, nt=50, nab=8),
    # not eligible (odd nz tiles, other orders): register-blocked kernels only
    dict(nd=3, freesurf=1, L=2, abs_type=1, src_type=100, nz=38, ny=29, nx=31, nt=80, nab=6),
    dict(nd=3, freesurf=0, L=1, abs_type=2, src_type=2, nz=70, ny=35, nx=22, nt=60, nab=5),
    dict(nd=3, freesurf=1, L=0, abs_type=1, src_type=0, nz=34, ny=18, nx=40, nt=60, nab=6, fdorder=12),
    dict(nd=3, freesurf=0, L=3, abs_type=1, src_type=100, nz=36, ny=20, nx=24, nt=60, nab=6, fdorder=4),
]


@pytest.mark.gpu
@pytest.mark.parametrize("kw", FAST_CASES, ids=lambda k: "-".join("%s%s" % (a, b) for a, b in k.items()))
def test_fast_3d_kernels_match_general(kw, cuda_device):
    """The vectorised, TMA-pipelined, streaming and register-blocked 3D
    kernels against the general ones (ragged tiles, CPML and taper, free
    surface, L = 0..3, FDORDER 4/8/12) and the oracle.  Eligible cases must
    actually take the vectorised (default) and TMA paths."""
    import dataclasses

    from oracle.oracle import Oracle
    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(**kw)
    outs = _outputs(3)
    res = {}
    for variant in ("fast", "tma", "stream", "register", "vector", "general"):
        ec = dataclasses.replace(engine_config(cfg), kernels=variant)
        plan = Plan(ec)
        plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
        eligible = kw.get("fdorder", 8) == 8 and kw["nz"] % 4 == 0
        assert plan.uses_tma == (variant == "tma" and eligible)
        want = {"fast": "vector" if eligible else "stream", "vector": "vector" if eligible else "stream",
                "tma": "tma" if eligible else "general", "stream": "stream", "register": "register",
                "general": "general"}[variant]
        assert plan.kernel_family == want, (variant, plan.kernel_family)
        res[variant] = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
    ora = Oracle(cfg)
    ora.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    ref = ora.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
    for n in outs:
        for v in ("fast", "tma", "stream", "register", "vector"):
            e_gen, e_ref = rel_l2(res[v][n], res["general"][n]), rel_l2(res[v][n], ref[n])
            assert e_gen < FAST_TOL and e_ref < FWD_TOL, (v, n, e_gen, e_ref)


ADJ_Q4_CASES = [
    dict(nd=3, freesurf=1, L=0, abs_type=1, src_type=100, nz=36, ny=30, nx=34, nt=80, nab=8),
    dict(nd=3, freesurf=0, L=2, abs_type=1, src_type=2, nz=40, ny=26, nx=30, nt=80, nab=6),
    dict(nd=3, freesurf=1, L=1, abs_type=2, src_type=0, nz=36, ny=28, nx=26, nt=80, nab=6),
    dict(nd=3, freesurf=0, L=3, abs_type=1, src_type=100, nz=44, ny=24, nx=28, nt=60, nab=8),
    dict(nd=3, freesurf=0, L=0, abs_type=1, src_type=1, nz=20, ny=24, nx=28, nt=60, nab=8),
]


@pytest.mark.gpu
@pytest.mark.parametrize("kw", ADJ_Q4_CASES, ids=lambda k: "-".join("%s%s" % (a, b) for a, b in k.items()))
def test_vectorised_adjoint_matches_general(kw, cuda_device):
    """The 4-cell vectorised 3D adjoint kernels (default) against the
    one-cell kernels on the same adjoint sources: gradients and the final
    adjoint and reconstructed fields; the gradient also against the oracle."""
    import dataclasses

    from oracle.oracle import Oracle
    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(**kw)
    outs = ["vx", "vy", "vz"]
    plans = {}
    for variant in ("fast", "general"):
        plan = Plan(dataclasses.replace(engine_config(cfg), kernels=variant))
        plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
        plans[variant] = plan
    assert plans["fast"].kernel_family == "vector"
    d = plans["general"].forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
    plans["fast"].forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
    n = plans["fast"].nvol
    # the forward fields at the last step: the scale of the reconstruction,
    # which backpropagates them to ~0 at t = 0
    scale = [float(np.linalg.norm(plans["general"].debug_array(0, i, n).astype(np.float64))) for i in range(9)]
    res = {k: (0.3 * v).astype(np.float32) for k, v in d.items()}
    g = {}
    for variant, plan in plans.items():
        plan.zero_gradient()
        plan.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], res)
        g[variant] = plan.gradient(transform=False)
    for k in g["general"]:
        ref = g["general"][k]
        assert np.abs(ref).max() > 0, k
        assert rel_l2(g["fast"][k], ref) < 2e-5, (k, rel_l2(g["fast"][k], ref))
    for i in range(9):
        a = plans["fast"].debug_array(1, i, n)
        b = plans["general"].debug_array(1, i, n)
        assert rel_l2(a, b) < 2e-5, ("adjoint", i)
    for i in range(9):
        # reconstructed forward fields, relative to their size before the
        # backpropagation: the CPML multiplies by 1/K in the 4-cell kernels
        # and divides by K in the one-cell ones, so the two runs differ by
        # roundings, and the residual the reconstruction leaves at t = 0 is
        # itself of rounding size
        a = plans["fast"].debug_array(0, i, n).astype(np.float64)
        b = plans["general"].debug_array(0, i, n).astype(np.float64)
        assert scale[i] > 0
        e = float(np.linalg.norm(a - b)) / max(float(np.linalg.norm(b)), scale[i])
        assert e < 2e-5, ("reconstructed", i, e)
    if cfg["L"]:
        # the reference's viscoelastic backpropagation is unstable
        # (update_adjs2D.cl:232): rounding differences grow, so the
        # oracle comparison is made for elastic media
        return
    ora = Oracle(cfg)
    ora.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    ora.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
    ora.clear_gradients()
    ora.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], res)
    og = ora.gradients()
    for ours, theirs in (("M", "rawM"), ("mu", "rawmu"), ("rho", "rawrho")):
        assert rel_l2(g["fast"][ours], og[theirs]) < GRAD_TOL, ours


OTHER_PHYSICS = [
    dict(nd=22, freesurf=0, L=0, abs_type=1, src_type=3),
    dict(nd=22, freesurf=0, L=1, abs_type=2, src_type=3),
    dict(nd=22, freesurf=0, L=0, abs_type=1, src_type=0, fdorder=4),
    dict(nd=21, freesurf=0, L=0, abs_type=1, src_type=1),
    dict(nd=21, freesurf=1, L=0, abs_type=2, src_type=1),
    dict(nd=21, freesurf=0, L=0, abs_type=1, src_type=1, fdorder=2),
]


@pytest.mark.gpu
@pytest.mark.parametrize("kw", OTHER_PHYSICS, ids=lambda k: "-".join("%s%s" % (a, b) for a, b in k.items()))
def test_acoustic_and_sh_forward_match_oracle(kw, cuda_device):
    """2D acoustic (ND=22) and SH (ND=21) forward modelling."""
    from oracle.oracle import Oracle
    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(**kw)
    outs = ["vx", "vz", "p"] if cfg["nd"] == 22 else ["vy", "sxy", "syz"]
    vp = model["vp"] if cfg["nd"] != 21 else None
    vs = model["vs"] if cfg["nd"] != 22 else None
    ora = Oracle(cfg)
    assert ora.set_model(vp, vs, model["rho"], model["taup"], model["taus"]) == 0
    ref = ora.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
    plan = Plan(engine_config(cfg))
    plan.set_model(vp, vs, model["rho"], model["taup"], model["taus"])
    got = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
    for n in outs:
        assert np.abs(ref[n]).max() > 0, n
        assert rel_l2(got[n], ref[n]) < FWD_TOL, (n, rel_l2(got[n], ref[n]))


FP16_CASES = [
    dict(nd=3, freesurf=1, L=0, abs_type=1, src_type=100, nz=40, ny=36, nx=44, nt=150, nab=8),
    dict(nd=3, freesurf=1, L=2, abs_type=1, src_type=2, nz=40, ny=36, nx=44, nt=150, nab=8),
    dict(nd=3, freesurf=0, L=1, abs_type=2, src_type=0, nz=36, ny=30, nx=40, nt=150, nab=8, fdorder=4),
    dict(nd=3, freesurf=1, L=2, abs_type=1, src_type=100, nz=38, ny=30, nx=34, nt=150, nab=8),
]


@pytest.mark.gpu
@pytest.mark.parametrize("kw", FP16_CASES, ids=lambda k: "-".join("%s%s" % (a, b) for a, b in k.items()))
def test_fp16_field_storage_against_fp32(kw, cuda_device):
    """Wave fields and memory variables stored in FP16 (power-of-two scaled,
    FP32 arithmetic) against the FP32 run: the reference's own criterion for
    its FP16 modes, sum (d - r)^2 / sum r^2 < 1e-3 over all outputs
    (test_consistency.py)."""
    import dataclasses

    from seiscl_b200.engine import Plan, SeisCLEngineError

    cfg, model, acq = make_case(**kw)
    outs = _outputs(3)
    res = {}
    for prec in ("fp32", "fp16"):
        plan = Plan(dataclasses.replace(engine_config(cfg), field_precision=prec))
        plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
        res[prec] = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
        if prec == "fp16":
            eligible = kw.get("fdorder", 8) == 8 and kw["nz"] % 4 == 0
            assert plan.kernel_family == ("vector" if eligible else "stream")
            with pytest.raises(SeisCLEngineError):   # the fields really are FP16
                plan.debug_array(0, 0, plan.nvol)
            with pytest.raises(SeisCLEngineError):   # forward modelling only
                plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
    # summed over all recorded outputs, as test_consistency.py does (a single
    # component can be ~0 by symmetry, e.g. vy in the source's plane)
    num = sum(float(((res["fp16"][n].astype(np.float64) - res["fp32"][n]) ** 2).sum()) for n in outs)
    den = sum(float((res["fp32"][n].astype(np.float64) ** 2).sum()) for n in outs)
    assert den > 0
    assert num / den < 1e-3, num / den


FP16_MEM_CASES = [
    dict(nd=3, freesurf=1, L=2, abs_type=1, src_type=2, nz=40, ny=36, nx=44, nt=150, nab=8, seed=84),
    dict(nd=3, freesurf=0, L=1, abs_type=2, src_type=100, nz=36, ny=30, nx=40, nt=150, nab=8, seed=85),
    dict(nd=3, freesurf=1, L=3, abs_type=1, src_type=100, nz=44, ny=26, nx=30, nt=150, nab=6, seed=86),
]


@pytest.mark.gpu
@pytest.mark.parametrize("kw", FP16_MEM_CASES, ids=["force_fs_L2", "taper_L1", "fs_L3"])
def test_fp16_memory_variables_against_fp32(kw, cuda_device):
    """Memory variables alone stored in FP16 (times a power of two set per
    shot), wave fields FP32: within 1e-3 relative L2 of the FP32 run and of
    the oracle over all outputs; the 4-cell kernels run it (free surface
    folded into the stress update, and the separate surface kernel of the
    kernel timings); what needs FP32 memory variables refuses the plan."""
    import dataclasses

    from oracle.oracle import Oracle
    from seiscl_b200.engine import Plan, SeisCLEngineError

    cfg, model, acq = make_case(**kw)
    outs = _outputs(3)
    res = {}
    for prec in ("fp32", "fp16_mem"):
        plan = Plan(dataclasses.replace(engine_config(cfg), field_precision=prec))
        plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
        res[prec] = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
        if prec == "fp16_mem":
            assert plan.kernel_family == "vector"
            assert np.isfinite(plan.debug_array(0, 0, plan.nvol)).all()   # wave fields stay FP32
            with pytest.raises(SeisCLEngineError):   # the memory variables are FP16
                plan.debug_array(2, 0, plan.nvol * cfg["L"])
            with pytest.raises(SeisCLEngineError):   # forward modelling only
                plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
            assert all(t >= 0 for t in plan.bench_kernels(1))
    ora = Oracle(cfg)
    ora.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    ref = ora.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
    ora.close()

    def joint(a, b):
        num = sum(float(((a[n].astype(np.float64) - b[n]) ** 2).sum()) for n in outs)
        den = sum(float((b[n].astype(np.float64) ** 2).sum()) for n in outs)
        assert den > 0
        return float(np.sqrt(num / den))

    e32, eora = joint(res["fp16_mem"], res["fp32"]), joint(res["fp16_mem"], ref)
    print("FP16 memory variables: rel L2 %.3g against FP32, %.3g against the oracle" % (e32, eora))
    assert e32 < 1e-3 and eora < 1e-3, (e32, eora)


FP16_2D_CASES = [
    dict(nd=2, freesurf=1, L=0, abs_type=1, src_type=100, nt=300, seed=81),
    dict(nd=2, freesurf=1, L=2, abs_type=1, src_type=2, nt=300, seed=82, fdorder=4),
    dict(nd=2, freesurf=0, L=1, abs_type=2, src_type=0, nt=300, seed=83, nz=70, nx=60),
]


@pytest.mark.gpu
@pytest.mark.parametrize("kw", FP16_2D_CASES, ids=["psv_fs", "psv_visco_o4", "psv_taper"])
def test_fp16_2d_field_storage_against_fp32(kw, cuda_device):
    """2D P-SV wave fields and memory variables stored in FP16 (power-of-two
    scaled, FP32 arithmetic) against the FP32 run, with the reference's
    criterion for its FP16 modes (sum (d - r)^2 / sum r^2 < 1e-3 over all
    outputs, test_consistency.py); the two-launch steps and the one-launch-
    per-kernel path agree in FP16 too; boundary saving is refused."""
    import dataclasses

    from seiscl_b200.engine import Plan, SeisCLEngineError

    cfg, model, acq = make_case(**kw)
    outs = ["vx", "vz", "p"]
    res = {}
    for prec, kern in (("fp32", "fast"), ("fp16", "fast"), ("fp16", "general")):
        plan = Plan(dataclasses.replace(engine_config(cfg), field_precision=prec, kernels=kern))
        plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
        res[(prec, kern)] = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
        if prec == "fp16" and kern == "fast":
            with pytest.raises(SeisCLEngineError):   # the fields really are FP16
                plan.debug_array(0, 0, plan.nvol)
            with pytest.raises(SeisCLEngineError):   # forward modelling only
                plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
        plan.close()
    ref, half = res[("fp32", "fast")], res[("fp16", "fast")]
    num = sum(float(((half[n].astype(np.float64) - ref[n]) ** 2).sum()) for n in outs)
    den = sum(float((ref[n].astype(np.float64) ** 2).sum()) for n in outs)
    assert den > 0
    print("FP16-2D %s energy ratio %.3g" % (kw, num / den))
    assert num / den < 1e-3, num / den
    for n in outs:
        assert rel_l2(res[("fp16", "general")][n], half[n]) < 1e-6, n


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(nd=2, freesurf=1, L=1, abs_type=1, src_type=100, nt=120),
                                dict(nd=3, freesurf=1, L=2, abs_type=1, src_type=2, nz=36, ny=30, nx=34, nt=60,
                                     nab=8)],
                         ids=["2d", "3d"])
def test_loop_graphs_match_direct_launches(kw, cuda_device):
    """Time loops replayed from captured CUDA graphs give the same bits as
    direct launches, including a second shot with new sources and data that
    reuses the captured graphs, and the gradient of both shots."""
    import dataclasses

    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(**kw)
    outs = _outputs(cfg["nd"])
    shots = [acq, dict(acq, src_pos=acq["src_pos"] + np.array([[30.0, 0, 10.0, 1, 0]], np.float32),
                       src=(0.7 * acq["src"]).astype(np.float32))]
    got = {}
    for mode in ("always", "never"):
        plan = Plan(dataclasses.replace(engine_config(cfg), loop_graphs=mode))
        plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
        plan.zero_gradient()
        seis = []
        for a in shots:
            d = plan.forward(a["src_pos"], a["src"], a["rec_pos"], outs, save_boundaries=True)
            seis.append(d)
            plan.adjoint(a["src_pos"], a["src"], a["rec_pos"],
                         {k: (0.3 * v).astype(np.float32) for k, v in d.items() if k != "p"})
        got[mode] = (seis, plan.gradient(transform=False))
    for s_a, s_b in zip(got["always"][0], got["never"][0]):
        for k in s_a:
            assert np.array_equal(s_a[k], s_b[k]), k
    for k in got["always"][1]:
        assert np.array_equal(got["always"][1][k], got["never"][1][k]), k


HESS_CASES = [
    (dict(nd=2, freesurf=1, L=0, abs_type=1, src_type=100), dict(hout=1)),
    (dict(nd=2, freesurf=0, L=0, abs_type=2, src_type=2), dict(hout=1, restype=1)),
    (dict(nd=2, freesurf=1, L=0, abs_type=1, src_type=100, nt=160), dict(hout=1, back_prop_type=2,
                                                                       gradfreqs=[10.0, 18.0])),
    (dict(nd=2, freesurf=0, L=1, abs_type=1, src_type=100, nt=160), dict(hout=1, back_prop_type=2,
                                                                       gradfreqs=[12.0, 20.0])),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", HESS_CASES, ids=lambda c: "-".join("%s%s" % kv for kv in c[1].items()
                                                                  if kv[0] != "gradfreqs"))
def test_hessian_matches_oracle(case, cuda_device):
    """The approximate Hessian (HOUT) of the CUDA path against the oracle:
    raw accumulators and, for the boundary-saving gradient, the transformed
    Hessian."""
    import dataclasses

    from oracle.oracle import Oracle
    from seiscl_b200.engine import Plan

    kw, extra = case
    cfg, model, acq = make_case(**kw)
    cfg.update(extra)
    ora = Oracle(cfg)
    ora.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    ec = dataclasses.replace(engine_config(cfg), hout=1, restype=extra.get("restype", 0),
                             back_prop_type=extra.get("back_prop_type", 1), gradfreqs=tuple(extra.get("gradfreqs", ())))
    plan = Plan(ec)
    plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    outs = ["vx", "vz"]
    d = ora.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
    plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
    res = {k: (0.3 * v).astype(np.float32) for k, v in d.items()}
    ora.clear_gradients()
    ora.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], res)
    plan.zero_gradient()
    plan.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], res)
    dft = extra.get("back_prop_type") == 2
    raw_o = ora.hessians(transform=False)
    raw_e = plan.hessian(transform=False)
    names = ("vp", "vs", "rho") if dft else ("M", "mu", "rho")
    pairs = list(zip(names, ("M", "mu", "rho")))
    if dft and cfg["L"]:
        pairs += [("taup", "taup"), ("taus", "taus")]
    for ours, theirs in pairs:
        ref = raw_o[theirs]
        if np.abs(ref).max() == 0:   # Hrho of the boundary-saving form stays zero
            assert np.abs(raw_e[ours]).max() == 0, ours
            continue
        assert rel_l2(raw_e[ours], ref) < GRAD_TOL, (ours, rel_l2(raw_e[ours], ref))
    if not dft:
        tr_o = ora.hessians(transform=True)
        tr_e = plan.hessian(transform=True)
        for k in ("vp", "vs", "rho"):
            if np.abs(tr_o[k]).max() > 0:
                assert rel_l2(tr_e[k], tr_o[k]) < GRAD_TOL, (k, rel_l2(tr_e[k], tr_o[k]))


FUSED_2D_CASES = [
    dict(nd=2, freesurf=1, L=0, abs_type=1, src_type=100, nt=150, seed=61),
    dict(nd=2, freesurf=1, L=2, abs_type=1, src_type=2, nt=150, seed=62, fdorder=4),
    dict(nd=2, freesurf=0, L=1, abs_type=2, src_type=0, nt=150, seed=63, nz=70, nx=45),
    dict(nd=22, freesurf=0, L=0, abs_type=1, src_type=3, nt=150, seed=64),
    dict(nd=22, freesurf=0, L=1, abs_type=2, src_type=3, nt=150, seed=65, fdorder=6),
]


@pytest.mark.gpu
@pytest.mark.parametrize("kw", FUSED_2D_CASES, ids=["psv_fs", "psv_visco_o4", "psv_taper", "acoustic",
                                                     "acoustic_visco_o6"])
def test_fused_2d_steps_match_separate_launches(kw, cuda_device):
    """2D modelling runs two launches per step (the stress update carries the
    free surface, the receivers of the step and the sources of the next);
    the general path runs one launch per reference kernel.  Same bits, with
    two sources in one cell, a receiver on a source cell and a second shot
    that replays the captured loop."""
    import dataclasses

    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(**kw)
    outs = ["vx", "vz", "p"]
    vs = None if cfg["nd"] == 22 else model["vs"]
    sp = np.concatenate([acq["src_pos"], acq["src_pos"]])
    src = np.concatenate([acq["src"], (0.5 * acq["src"][:, ::-1]).copy()]).astype(np.float32)
    rp = acq["rec_pos"].copy()
    rp[0, 0], rp[0, 2] = sp[0, 0], sp[0, 2]
    shots = [(sp, src, rp), (acq["src_pos"] + np.array([[40.0, 0, 10.0, 1, 0]], np.float32), acq["src"], rp)]
    got = {}
    for kern in ("fast", "general"):
        plan = Plan(dataclasses.replace(engine_config(cfg), kernels=kern))
        plan.set_model(model["vp"], vs, model["rho"], model["taup"], model["taus"])
        got[kern] = [plan.forward(s, w, r, outs) for s, w, r in shots]
        plan.close()
    for a, b in zip(got["fast"], got["general"]):
        for k in outs:
            assert np.abs(b[k]).max() > 0, k
            assert np.array_equal(a[k], b[k]), (k, float(np.abs(a[k] - b[k]).max()))


BATCH_CASES = [
    dict(nd=2, freesurf=1, L=0, abs_type=1, src_type=100, nt=150, seed=91),
    dict(nd=2, freesurf=1, L=2, abs_type=1, src_type=2, nt=150, seed=92, fdorder=4),
    dict(nd=2, freesurf=0, L=0, abs_type=2, src_type=0, nt=150, seed=93),
    dict(nd=22, freesurf=0, L=1, abs_type=1, src_type=3, nt=150, seed=94),
]


@pytest.mark.gpu
@pytest.mark.parametrize("kw", BATCH_CASES, ids=["psv_fs", "psv_visco", "psv_taper", "acoustic"])
def test_batched_shots_match_single_runs(kw, cuda_device):
    """Shots advanced together (one launch per kernel and step for all of
    them) give each shot the seismograms it gets alone, bit for bit, and the
    gradient of the batch is the sum of the shots' gradients."""
    import dataclasses

    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(**kw)
    outs = ["vx", "vz", "p"]
    vs = None if cfg["nd"] == 22 else model["vs"]
    shots = []
    for j in range(3):
        sp = acq["src_pos"] + np.array([[20.0 * j, 0, 10.0 * (j % 2), j, 0]], np.float32)
        rp = acq["rec_pos"][j:] if j < 2 else acq["rec_pos"]   # ragged receiver counts
        shots.append((sp, ((1.0 + 0.3 * j) * acq["src"]).astype(np.float32), rp))
    one = Plan(engine_config(cfg))
    one.set_model(model["vp"], vs, model["rho"], model["taup"], model["taus"])
    many = Plan(dataclasses.replace(engine_config(cfg), batch=4))
    many.set_model(model["vp"], vs, model["rho"], model["taup"], model["taus"])
    grad = cfg["nd"] == 2
    ref = [one.forward(sp, src, rp, outs, save_boundaries=False) for sp, src, rp in shots]
    got = many.forward_batch(shots, outs)
    for r, g in zip(ref, got):
        for k in outs:
            assert np.abs(r[k]).max() > 0, k
            assert np.array_equal(r[k], g[k]), (k, float(np.abs(r[k] - g[k]).max()))
    assert np.array_equal(many.forward_batch(shots[1:2], outs)[0]["vx"], ref[1]["vx"])
    if not grad:
        return
    gouts = ["vx", "vz"]
    one.zero_gradient()
    for sp, src, rp in shots:
        d = one.forward(sp, src, rp, gouts, save_boundaries=True)
        one.adjoint(sp, src, rp, {k: (0.3 * v).astype(np.float32) for k, v in d.items()})
    many.zero_gradient()
    d = many.forward_batch(shots, gouts, save_boundaries=True)
    many.adjoint_batch(shots, [{k: (0.3 * v).astype(np.float32) for k, v in di.items()} for di in d])
    g1, gb = one.gradient(transform=False), many.gradient(transform=False)
    for k in ("M", "mu", "rho"):
        assert np.abs(g1[k]).max() > 0, k
        assert rel_l2(gb[k], g1[k]) < 1e-6, (k, rel_l2(gb[k], g1[k]))


BATCH3D_CASES = [
    dict(nd=3, freesurf=1, L=0, abs_type=1, src_type=100, nz=36, ny=30, nx=34, nt=80, nab=8, seed=95),
    dict(nd=3, freesurf=1, L=2, abs_type=1, src_type=2, nz=36, ny=30, nx=34, nt=80, nab=8, seed=96, fdorder=4),
    dict(nd=3, freesurf=0, L=1, abs_type=2, src_type=0, nz=38, ny=30, nx=34, nt=80, nab=8, seed=97),
]


@pytest.mark.gpu
@pytest.mark.parametrize("kw", BATCH3D_CASES, ids=["vector", "stream_o4", "general_taper"])
def test_batched_3d_shots_match_single_runs(kw, cuda_device):
    """3D shots advanced together: the 4-cell (8th order, nz % 4 == 0),
    streaming (4th order) and one-cell (nz % 4 != 0) kernels, forward bit
    for bit against single runs, the gradient of the batch against the sum
    over single runs."""
    import dataclasses

    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(**kw)
    outs = ["vx", "vy", "vz", "p"]
    shots = []
    for j in range(3):
        sp = acq["src_pos"] + np.array([[20.0 * j, 10.0 * j, 0, j, 0]], np.float32)
        shots.append((sp, ((1.0 + 0.3 * j) * acq["src"]).astype(np.float32), acq["rec_pos"][j:]))
    one = Plan(engine_config(cfg))
    one.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    many = Plan(dataclasses.replace(engine_config(cfg), batch=3))
    many.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    assert one.kernel_family == many.kernel_family
    ref = [one.forward(sp, src, rp, outs) for sp, src, rp in shots]
    got = many.forward_batch(shots, outs)
    for r, g in zip(ref, got):
        for k in outs:
            assert np.abs(r[k]).max() > 0, k
            assert np.array_equal(r[k], g[k]), (k, float(np.abs(r[k] - g[k]).max()))
    gouts = ["vx", "vz"]
    one.zero_gradient()
    for sp, src, rp in shots:
        d = one.forward(sp, src, rp, gouts, save_boundaries=True)
        one.adjoint(sp, src, rp, {k: (0.3 * v).astype(np.float32) for k, v in d.items()})
    many.zero_gradient()
    d = many.forward_batch(shots, gouts, save_boundaries=True)
    many.adjoint_batch(shots, [{k: (0.3 * v).astype(np.float32) for k, v in di.items()} for di in d])
    g1, gb = one.gradient(transform=False), many.gradient(transform=False)
    for k in ("M", "mu", "rho"):
        assert np.abs(g1[k]).max() > 0, k
        assert rel_l2(gb[k], g1[k]) < 1e-6, (k, rel_l2(gb[k], g1[k]))


@pytest.mark.gpu
@pytest.mark.parametrize("nd", [2, 3])
def test_unstable_run_is_reported(nd, cuda_device, monkeypatch):
    """A time step far above the CFL limit (the set-up check bypassed through
    its test hook) diverges; the forward run returns SFD_ERR_UNSTABLE naming
    a checked step at most 64 steps after the field first stops being
    finite, and the adjoint of a finite forward run with non-finite
    residuals does the same."""
    from seiscl_b200.engine import Plan, SeisCLEngineError

    monkeypatch.setenv("SEISCL_B200_UNCHECKED_CFL", "1")
    kw = dict(nd=nd, nt=300, nz=32, nx=36, ny=28, nab=8) if nd == 3 else dict(nd=nd, nt=300)
    cfg, model, acq = make_case(**kw)
    cfg["dt"] = 4e-3   # ~3x the stability limit
    plan = Plan(engine_config(cfg))
    plan.set_model(model["vp"], model["vs"], model["rho"])
    with pytest.raises(SeisCLEngineError) as e:
        plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], ["vx"])
    assert e.value.code == -6
    assert "unstable" in str(e.value)
    step = int(str(e.value).rsplit("step", 1)[1].split()[0])
    assert 0 <= step < cfg["nt"]
    # the adjoint reports it too: a finite forward, non-finite residuals
    cfg2, model2, acq2 = make_case(**kw)
    plan2 = Plan(engine_config(cfg2))
    plan2.set_model(model2["vp"], model2["vs"], model2["rho"])
    d = plan2.forward(acq2["src_pos"], acq2["src"], acq2["rec_pos"], ["vx"], save_boundaries=True)
    res = {"vx": np.full_like(d["vx"], np.nan)}
    with pytest.raises(SeisCLEngineError) as e2:
        plan2.adjoint(acq2["src_pos"], acq2["src"], acq2["rec_pos"], res)
    assert e2.value.code == -6


FUSED_CASES = [
    # ragged tiles in every direction (nz not a multiple of 32, ny of 8, nx of 8)
    dict(nd=3, freesurf=1, L=2, abs_type=1, src_type=2, nz=36, ny=34, nx=38, nt=120, nab=8),
    dict(nd=3, freesurf=1, L=0, abs_type=1, src_type=100, nz=64, ny=16, nx=24, nt=100, nab=8),
    dict(nd=3, freesurf=0, L=1, abs_type=2, src_type=1, nz=40, ny=21, nx=17, nt=100, nab=6),
    dict(nd=3, freesurf=1, L=3, abs_type=1, src_type=0, nz=100, ny=12, nx=19, nt=80, nab=4),
    dict(nd=3, freesurf=0, L=2, abs_type=1, src_type=100, nz=32, ny=40, nx=44, nt=80, nab=10),
]


@pytest.mark.gpu
@pytest.mark.parametrize("kw", FUSED_CASES, ids=lambda k: "-".join("%s%s" % (a, b) for a, b in k.items()))
def test_fused_3d_step_matches_separate_kernels(kw, cuda_device):
    """The fused 3D step (velocity, stress, memory variables and free surface
    in one launch per step, CTAs ordered by tickets and synchronised by
    neighbour flags) against the same 4-cell kernels launched separately:
    the same per-cell arithmetic, so the seismograms and every final wave
    field and memory variable agree to rounding (the compiler may contract
    a product into an FMA differently in the two kernels: 1e-6 relative for
    seismograms, 1e-5 for fields after up to 120 steps); and against the
    oracle."""
    import dataclasses

    from oracle.oracle import Oracle
    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(**kw)
    outs = _outputs(3)
    res, fields = {}, {}
    for variant in ("fused", "vector"):
        plan = Plan(dataclasses.replace(engine_config(cfg), kernels=variant))
        plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
        assert plan.fused_step == (variant == "fused")
        res[variant] = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
        nv = plan.nvol
        fields[variant] = [plan.debug_array(0, i, nv) for i in range(9)]
        if cfg["L"]:
            fields[variant] += [plan.debug_array(2, i, nv * cfg["L"]) for i in range(6)]
    for n in outs:
        assert np.abs(res["vector"][n]).max() > 0
        assert rel_l2(res["fused"][n], res["vector"][n]) < 1e-6, n
    errs = [rel_l2(a, b) for a, b in zip(fields["fused"], fields["vector"])]
    assert max(errs) < 1e-5, errs
    ora = Oracle(cfg)
    ora.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    ref = ora.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
    for n in outs:
        assert rel_l2(res["fused"][n], ref[n]) < FWD_TOL, n


@pytest.mark.gpu
@pytest.mark.parametrize("kw", FUSED_CASES, ids=lambda k: "-".join("%s%s" % (a, b) for a, b in k.items()))
def test_async_velocity_kernel_matches_vector(kw, cuda_device):
    """The cp.async-staged velocity update (stress operands copied into a
    shared-memory ring, kernels "async") against the 4-cell kernel reading
    them from global memory: the same values in the same operation order, so
    identical seismograms and fields (ragged tiles in z, y and x)."""
    import dataclasses

    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(**kw)
    outs = _outputs(3)
    res, fields = {}, {}
    for variant in ("async", "vector"):
        plan = Plan(dataclasses.replace(engine_config(cfg), kernels=variant))
        plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
        res[variant] = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
        fields[variant] = [plan.debug_array(0, i, plan.nvol) for i in range(9)]
    for n in outs:
        assert np.abs(res["vector"][n]).max() > 0
        assert np.array_equal(res["async"][n], res["vector"][n]), (n, rel_l2(res["async"][n], res["vector"][n]))
    for a, b in zip(fields["async"], fields["vector"]):
        assert np.array_equal(a, b), rel_l2(a, b)


@pytest.mark.gpu
def test_concurrent_3d_plans_are_deterministic(cuda_device):
    """Single-shot 3D modelling plans on worker threads, each plan on its own
    stream (the stress update, sources and receivers launched with
    programmatic stream serialization, kernels of different plans sharing
    the GPU): every run equals the same plan's run alone, bit for bit (FP32,
    FP16 memory variables and FP16 storage, elastic and viscoelastic)."""
    import dataclasses
    import threading

    from seiscl_b200.engine import Plan

    cases = [(dict(nd=3, freesurf=1, L=2, abs_type=1, src_type=2, nz=40, ny=36, nx=44, nt=120, nab=8, seed=91),
              "fp32"),
             (dict(nd=3, freesurf=0, L=1, abs_type=1, src_type=100, nz=36, ny=30, nx=40, nt=120, nab=8, seed=92),
              "fp16_mem"),
             (dict(nd=3, freesurf=1, L=0, abs_type=1, src_type=100, nz=44, ny=28, nx=32, nt=120, nab=6, seed=93),
              "fp16"),
             (dict(nd=3, freesurf=1, L=3, abs_type=2, src_type=0, nz=40, ny=26, nx=30, nt=120, nab=6, seed=94), "fp32")]
    jobs = []
    for kw, prec in cases:
        cfg, model, acq = make_case(**kw)
        jobs.append((dataclasses.replace(engine_config(cfg), field_precision=prec), model, acq))
    outs = _outputs(3)

    def run(job, reps):
        cfg, model, acq = job
        plan = Plan(cfg)
        plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
        got = [plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs) for _ in range(reps)]
        plan.close()
        return got

    alone = [run(j, 1)[0] for j in jobs]
    results, errors = [None] * len(jobs), []

    def worker(i):
        try:
            results[i] = run(jobs[i], 3)   # the second and third runs replay captured graphs
        except Exception as e:             # surfaced below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(len(jobs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for i, runs in enumerate(results):
        for r in runs:
            for n in outs:
                assert np.abs(alone[i][n]).max() > 0, (i, n)
                assert np.array_equal(r[n], alone[i][n]), (i, n, rel_l2(r[n], alone[i][n]))
