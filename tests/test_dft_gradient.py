"""DFT gradient (SeisCL's BACK_PROP_TYPE=2).

CPU (oracle): the forward transform at a receiver cell is the DFT of the
recorded trace, and the gradient behaves physically (elastic: the same image
as the boundary-saving gradient; weak attenuation: the same image as the
elastic DFT gradient).  The oracle itself is pinned to the reference's
kernels and calc_grad by tests/test_oracle_pin.py.

GPU: transforms and gradients of the CUDA path against the oracle, shot
accumulation, the call-order errors, and the receiver-trace property on a
larger 3D grid.

Tolerances (relative L2): transforms 2e-5 (FP32 fields with FMA, FMA in the
accumulation); gradients 2e-4 (as the boundary-saving gradient: FP64 sums
here, FP32 in the reference).
"""
import numpy as np
import pytest

from tests._cases import engine_config, make_case, rel_l2

DFT_TOL = 2e-5
GRAD_TOL = 2e-4
WAVE = {2: ["vx", "vz", "sxx", "szz", "sxz"], 3: ["vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "syz", "sxz"]}
MEM = {2: ["rxx", "rzz", "rxz"], 3: ["rxx", "ryy", "rzz", "rxy", "ryz", "rxz"]}


def crel(a, b):
    """Relative L2 of two complex arrays over real and imaginary parts."""
    return rel_l2(np.asarray(a, np.complex64).view(np.float32), np.asarray(b, np.complex64).view(np.float32))


def _inputs(model, param_type):
    vp, vs, rho = model["vp"], model["vs"], model["rho"]
    if param_type == 1:
        return (rho * vp * vp).astype(np.float32), (rho * vs * vs).astype(np.float32), rho
    if param_type == 2:
        return (rho * vp).astype(np.float32), (rho * vs).astype(np.float32), rho
    return vp, vs, rho


def _factors(info, nt_samples, dt_lit):
    """DTNYQ*DT*exp(-i 2 pi k n / NTNYQ) for every sample n, in FP64."""
    n = np.arange(nt_samples)
    k = info["gradfreqsn"].astype(np.float64)[:, None]
    return info["dtnyq"] * dt_lit * np.exp(-2j * np.pi * k * n[None, :] / info["ntnyq"])


def _receiver_dft(seis, info, tmin, tmax, dt_lit):
    """The transform a receiver cell should hold: the state after t steps is
    the sample recorded at step t - 1 (zero at t = 0)."""
    ts = np.arange(tmin, tmax, info["dtnyq"])
    x = np.zeros((seis.shape[0], len(ts)))
    ok = ts >= 1
    x[:, ok] = seis[:, ts[ok] - 1]
    return x @ _factors(info, len(ts), dt_lit).T  # [nrec][nfreqs]


def _rec_cells(o_or_plan, acq, nd, F, dh):
    rp = acq["rec_pos"]
    i = (rp[:, 0] / dh).astype(int) + F
    k = (rp[:, 2] / dh).astype(int) + F
    if nd == 3:
        j = (rp[:, 1] / dh).astype(int) + F
        return (i * o_or_plan.NYp + j) * o_or_plan.NZp + k
    return i * o_or_plan.NZp + k


def test_oracle_transform_is_dft_of_receiver_trace():
    from oracle.oracle import Oracle

    cfg, model, acq = make_case(nd=2, freesurf=1, L=1, nt=150, seed=21)
    cfg.update(back_prop_type=2, gradfreqs=[9.0, 16.0, 30.0], tmin=7)
    o = Oracle(cfg)
    assert o.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"]) == 0
    d = o.forward(acq["src_pos"], acq["src"], acq["rec_pos"], ["vx", "vz"], save_boundaries=True)
    info = o.dft_info()
    assert info["dtnyq"] == int(np.ceil(0.0156 / 30.0 / np.float32(1e-3)))
    dt_lit = float("%9.9f" % np.float32(cfg["dt"]))
    cells = _rec_cells(o, acq, 2, cfg["fdorder"] // 2, cfg["dh"])
    for name in ("vx", "vz"):
        want = _receiver_dft(d[name].astype(np.float64), info, 7, cfg["nt"], dt_lit)
        got = o.dft(0, "wave", name).reshape(len(info["gradfreqsn"]), -1)[:, cells].T
        assert rel_l2(got.real, want.real) < 1e-5 and rel_l2(got.imag, want.imag) < 1e-5, name


def _corr(a, b, nab):
    sl = (slice(nab, -nab), slice(nab, -nab))
    a = a[sl].ravel().astype(np.float64)
    b = b[sl].ravel().astype(np.float64)
    return np.corrcoef(a, b)[0, 1]


def test_oracle_dft_gradient_is_physical():
    """With all bins up to 40 Hz the elastic DFT gradient images like the
    boundary-saving one; with weak attenuation (tau = 0.01) like the elastic
    DFT gradient.  (The reference's boundary-saving viscoelastic gradient does
    not: its backpropagation is not stable, update_adjs2D.cl:232.)"""
    from oracle.oracle import Oracle

    grads = {}
    for L in (0, 1):
        cfg, model, acq = make_case(nd=2, freesurf=0, L=L, nt=400, seed=3, nz=60, nx=70)
        if L:
            model["taup"][:] = 0.01
            model["taus"][:] = 0.01
        for bp in ((1, 2) if L == 0 else (2,)):
            c = dict(cfg)
            c.update(back_prop_type=bp, gradfreqs=[2.4938 * k + 0.1 for k in range(1, 17)])
            o = Oracle(c)
            assert o.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"]) == 0
            d = o.forward(acq["src_pos"], acq["src"], acq["rec_pos"], ["vx", "vz"], save_boundaries=True)
            o.clear_gradients()
            o.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], {k: (0.3 * v).astype(np.float32) for k, v in d.items()})
            g = o.gradients() if bp == 1 else o.raw_gradients()
            grads[(L, bp)] = (g["vp"], g["vs"]) if bp == 1 else (g["M"], g["mu"])
    nab = cfg["nab"]
    for q in (0, 1):
        assert _corr(grads[(0, 1)][q], grads[(0, 2)][q], nab) > 0.99
        assert _corr(grads[(0, 2)][q], grads[(1, 2)][q], nab) > 0.999


# ------------------------------------------------------------------ GPU
DFT_CASES = [
    (dict(nd=2, freesurf=1, L=0, abs_type=1, src_type=100, nt=160, seed=31), [10.0, 18.0, 25.0], 0),
    (dict(nd=2, freesurf=0, L=2, abs_type=1, src_type=2, nt=160, seed=32), [12.0, 20.0], 2),
    (dict(nd=2, freesurf=0, L=1, abs_type=2, src_type=100, nt=160, seed=33), [15.0], 1),
    (dict(nd=3, freesurf=1, L=1, abs_type=1, src_type=100, nz=34, ny=30, nx=36, nt=90, nab=8, seed=34), [20.0, 35.0], 0),
    (dict(nd=3, freesurf=0, L=0, abs_type=1, src_type=2, nz=34, ny=30, nx=36, nt=90, nab=8, seed=35), [25.0], 2),
    # nz % 4 == 0: the 4-cell vectorised adjoint kernels in their DFT form
    (dict(nd=3, freesurf=0, L=2, abs_type=1, src_type=100, nz=36, ny=30, nx=32, nt=90, nab=8, seed=38), [20.0, 35.0], 1),
    (dict(nd=3, freesurf=1, L=0, abs_type=1, src_type=2, nz=40, ny=28, nx=30, nt=90, nab=6, seed=39), [25.0], 0),
]


def _pair(kw, freqs, pt, tmin=0):
    from oracle.oracle import Oracle
    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(**kw)
    cfg.update(back_prop_type=2, gradfreqs=freqs, param_type=pt, tmin=tmin)
    a, b, rho = _inputs(model, pt)
    ora = Oracle(cfg)
    assert ora.set_model(a, b, rho, model["taup"], model["taus"]) == 0
    ec = engine_config(cfg)
    ec.back_prop_type, ec.gradfreqs, ec.param_type, ec.tmin = 2, freqs, pt, tmin
    plan = Plan(ec)
    plan.set_model(a, b, rho, model["taup"], model["taus"])
    return cfg, acq, ora, plan


@pytest.mark.gpu
@pytest.mark.parametrize("case", DFT_CASES, ids=lambda c: "nd%d-L%d-pt%d" % (c[0]["nd"], c[0]["L"], c[2]))
def test_dft_gradient_matches_oracle(case, cuda_device):
    kw, freqs, pt = case
    cfg, acq, ora, plan = _pair(kw, freqs, pt)
    nd = cfg["nd"]
    outs = ["vx", "vy", "vz"] if nd == 3 else ["vx", "vz"]
    d_ref = ora.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
    d_gpu = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
    info = ora.dft_info()
    assert (plan.dtnyq, plan.ntnyq) == (info["dtnyq"], info["ntnyq"])
    for n in WAVE[nd]:
        assert crel(plan.dft(0, "wave", n), ora.dft(0, "wave", n)) < DFT_TOL, n
    res = {k: (0.3 * v).astype(np.float32) for k, v in d_ref.items()}
    ora.clear_gradients()
    ora.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], res)
    plan.zero_gradient()
    plan.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], res)
    for n in WAVE[nd]:
        ref = ora.dft(1, "wave", n)
        assert np.abs(ref).max() > 0, n
        assert crel(plan.dft(1, "wave", n), ref) < DFT_TOL, n
    if cfg["L"]:
        for n in MEM[nd]:
            for slot in (0, 1):
                assert crel(plan.dft(slot, "mem", n), ora.dft(slot, "mem", n)) < DFT_TOL, (slot, n)
    g_ref = ora.raw_gradients()
    g_gpu = plan.gradient()
    names = {0: ("vp", "vs", "rho"), 1: ("M", "mu", "rho"), 2: ("Ip", "Is", "rho")}[pt]
    pairs = list(zip(names, ("M", "mu", "rho")))
    if cfg["L"]:
        pairs += [("taup", "taup"), ("taus", "taus")]
    for ours, theirs in pairs:
        ref = g_ref[theirs]
        assert np.isfinite(g_gpu[ours]).all() and np.abs(ref).max() > 0, ours
        err = rel_l2(g_gpu[ours], ref)
        assert err < GRAD_TOL, (ours, err)


@pytest.mark.gpu
def test_dft_gradient_accumulates_over_shots(cuda_device):
    kw, freqs, pt = DFT_CASES[1]
    cfg, acq, ora, plan = _pair(kw, freqs, pt)
    shots = [acq, dict(acq, src_pos=acq["src_pos"] + np.array([[60.0, 0, 20.0, 1, 0]], np.float32))]
    plan.zero_gradient()
    single = []
    for a in shots:
        d = plan.forward(a["src_pos"], a["src"], a["rec_pos"], ["vx", "vz"], save_boundaries=True)
        plan.adjoint(a["src_pos"], a["src"], a["rec_pos"], {k: (0.3 * v).astype(np.float32) for k, v in d.items()})
    both = plan.gradient()
    for a in shots:
        plan.zero_gradient()
        d = plan.forward(a["src_pos"], a["src"], a["rec_pos"], ["vx", "vz"], save_boundaries=True)
        plan.adjoint(a["src_pos"], a["src"], a["rec_pos"], {k: (0.3 * v).astype(np.float32) for k, v in d.items()})
        single.append(plan.gradient())
    for k in both:
        assert rel_l2(both[k], single[0][k] + single[1][k]) < 1e-6, k


@pytest.mark.gpu
def test_dft_call_order_errors(cuda_device):
    from seiscl_b200.engine import Plan, SeisCLEngineError

    cfg, model, acq = make_case(nd=2, freesurf=0, L=0, nt=60, seed=36)
    ec = engine_config(cfg)
    p1 = Plan(ec)
    with pytest.raises(SeisCLEngineError):
        p1.set_gradfreqs([10.0])  # boundary-saving plan
    ec.back_prop_type = 2
    p2 = Plan(ec)
    p2.set_model(model["vp"], model["vs"], model["rho"])
    with pytest.raises(SeisCLEngineError):  # no frequencies yet
        p2.forward(acq["src_pos"], acq["src"], acq["rec_pos"], ["vx"], save_boundaries=True)
    for bad in ([], [0.0], [-1.0, 5.0], list(range(1, 18))):
        with pytest.raises(SeisCLEngineError):
            p2.set_gradfreqs(np.asarray(bad, np.float32))
    p2.set_gradfreqs([10.0])
    d = p2.forward(acq["src_pos"], acq["src"], acq["rec_pos"], ["vx"], save_boundaries=True)
    p2.set_gradfreqs([10.0, 20.0])  # invalidates the forward transforms
    with pytest.raises(SeisCLEngineError):
        p2.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], {"vx": d["vx"]})


@pytest.mark.gpu
def test_dft_receiver_property_3d(cuda_device):
    """On a 3D grid too large for the oracle: the device transform at each
    receiver cell equals the DFT of the device seismogram there."""
    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(nd=3, freesurf=1, L=2, nz=96, ny=96, nx=96, nt=300, nab=12, seed=37, src_type=100)
    ec = engine_config(cfg)
    ec.back_prop_type, ec.gradfreqs, ec.tmin = 2, [8.0, 15.0, 24.0], 11
    plan = Plan(ec)
    plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    d = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], ["vx", "vz"], save_boundaries=True)
    tmax = cfg["nt"]
    ntnyq = (tmax - 11) // plan.dtnyq + 1
    df = np.float32(1.0 / ntnyq / np.float32(cfg["dt"]) / plan.dtnyq)
    info = {"dtnyq": plan.dtnyq, "ntnyq": plan.ntnyq,
            "gradfreqsn": np.floor(np.float32([8.0, 15.0, 24.0]) / df).astype(np.float32)}
    assert plan.ntnyq == ntnyq
    dt_lit = float("%9.9f" % np.float32(cfg["dt"]))
    cells = _rec_cells(plan, acq, 3, cfg["fdorder"] // 2, cfg["dh"])
    for name in ("vx", "vz"):
        want = _receiver_dft(d[name].astype(np.float64), info, 11, tmax, dt_lit)
        got = plan.dft(0, "wave", name).reshape(3, -1)[:, cells].T
        assert rel_l2(got.real, want.real) < 1e-5 and rel_l2(got.imag, want.imag) < 1e-5, name
