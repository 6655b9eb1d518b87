"""Pins the CPU oracle (oracle/fdo_port.c) to the reference.

* Golden vectors in tests/golden/ were produced by the reference's own
  kernel sources compiled in place (tests/golden/make_golden.py); the port
  must reproduce them bit for bit.
* Where the reference tree is present, extra cases are compared live against
  an in-place build of the reference kernels.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from tests._cases import make_case

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
with open(os.path.join(GOLD, "index.json")) as f:
    INDEX = json.load(f)


def _input_hash(model, acq):
    h = hashlib.sha256()
    for d in (model, acq):
        for k in sorted(d):
            if d[k] is not None:
                h.update(k.encode())
                h.update(np.ascontiguousarray(d[k]).tobytes())
    return h.hexdigest()


def _run(kw, ref=False):
    from oracle.oracle import Oracle

    cfg, model, acq = make_case(**kw)
    o = Oracle(cfg, ref=ref)
    nd = cfg["nd"]
    assert o.set_model(model["vp"] if nd != 21 else None, model["vs"] if nd != 22 else None, model["rho"],
                       model["taup"], model["taus"]) == 0
    outs = {3: ["vx", "vy", "vz", "p"], 21: ["vy", "sxy", "syz"]}.get(nd, ["vx", "vz", "p"])
    if nd in (21, 22):
        return cfg, model, acq, o.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs), {}, o
    d = o.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
    res = {k: (0.3 * v).astype(np.float32) for k, v in d.items() if k != "p"}
    o.clear_gradients()
    o.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], res)
    return cfg, model, acq, d, o.gradients(), o


TIME_CASES = sorted(k for k, v in INDEX.items() if "extra" not in v)
DFT_CASES = sorted(k for k, v in INDEX.items() if "extra" in v)


@pytest.mark.parametrize("name", TIME_CASES)
def test_port_reproduces_golden(name):
    entry = INDEX[name]
    cfg, model, acq, d, g, _ = _run(entry["kwargs"])
    assert _input_hash(model, acq) == entry["input_sha256"]
    gold = np.load(os.path.join(GOLD, name + ".npz"))
    for k, v in d.items():
        assert np.array_equal(v, gold["seis_" + k]), k
    for k, v in g.items():
        if cfg["nd"] in (2, 21, 22):
            assert np.array_equal(v, gold["grad_" + k]), k
        else:
            v64 = v.astype(np.float64)
            assert np.array_equal(np.array([v64.sum(), (v64 * v64).sum(), np.abs(v64).max()]), gold["gradsum_" + k]), k


@pytest.mark.parametrize("name", DFT_CASES)
def test_port_reproduces_dft_golden(name):
    """DFT gradient (BACK_PROP_TYPE=2): seismograms and transforms bit for bit
    (the reference's adjoint kernels compiled with BACK_PROP_TYPE=2); the
    gradient within 1e-6 of the reference's calc_grad (src/calc_grad.c, whose
    float/double mix the restatement follows up to the order of a few
    products)."""
    from tests.golden.make_golden import run_dft

    entry = INDEX[name]
    cfg, model, acq, d, g, sums = run_dft(entry["kwargs"], entry["extra"], ref=False)
    assert _input_hash(model, acq) == entry["input_sha256"]
    gold = np.load(os.path.join(GOLD, name + ".npz"))
    for k, v in d.items():
        assert np.array_equal(v, gold["seis_" + k]), k
    for k, v in sums.items():
        assert np.array_equal(v, gold[k]), k
    for k, v in g.items():
        if cfg["nd"] == 2:
            ref = gold["grad_" + k]
            scale = np.abs(ref).max()
            assert np.abs(v - ref).max() <= 1e-6 * scale, k
        else:
            v64 = v.astype(np.float64)
            got = np.array([v64.sum(), (v64 * v64).sum(), np.abs(v64).max()])
            ref = gold["gradsum_" + k]
            assert np.allclose(got, ref, rtol=1e-5, atol=1e-6 * abs(ref[2]) * v.size), k


def _ref_available():
    from oracle import build

    return build.ref_available()


LIVE_2D_OTHER = [
    dict(nd=22, freesurf=0, L=0, abs_type=1, src_type=3, nt=80, seed=6),
    dict(nd=22, freesurf=0, L=2, abs_type=2, src_type=0, nt=80, seed=7),
    dict(nd=21, freesurf=0, L=0, abs_type=1, src_type=1, nt=80, seed=8),
    dict(nd=21, freesurf=0, L=0, abs_type=2, src_type=1, nt=80, seed=9, fdorder=2),
]


@pytest.mark.skipif(not _ref_available(), reason="reference tree not present")
@pytest.mark.parametrize("kw", LIVE_2D_OTHER, ids=lambda k: "-".join("%s%s" % (a, b) for a, b in k.items()))
def test_acoustic_sh_port_matches_reference_build(kw):
    """Acoustic (ND=22) and SH (ND=21) forward kernels, compiled in place."""
    from oracle.oracle import Oracle

    cfg, model, acq = make_case(**kw)
    outs = ["vx", "vz", "p"] if cfg["nd"] == 22 else ["vy", "sxy", "syz"]
    vp = model["vp"] if cfg["nd"] != 21 else None
    vs = model["vs"] if cfg["nd"] != 22 else None
    res = []
    for ref in (False, True):
        o = Oracle(cfg, ref=ref)
        assert o.set_model(vp, vs, model["rho"], model["taup"], model["taus"]) == 0
        res.append(o.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs))
    for k in outs:
        assert np.abs(res[0][k]).max() > 0
        assert np.array_equal(res[0][k], res[1][k]), k


LIVE = [
    dict(nd=2, freesurf=1, L=2, abs_type=1, src_type=0, nt=80, seed=3),
    dict(nd=2, freesurf=0, L=0, abs_type=1, src_type=100, fdorder=12, nz=50, nx=46, nt=80, seed=4),
    dict(nd=3, freesurf=0, L=1, abs_type=2, src_type=1, nz=30, ny=28, nx=32, nt=50, nab=6, seed=5),
]


@pytest.mark.skipif(not _ref_available(), reason="reference tree not present")
@pytest.mark.parametrize("kw", LIVE, ids=lambda k: "-".join("%s%s" % (a, b) for a, b in k.items()))
def test_port_matches_reference_build(kw):
    a = _run(kw, ref=False)
    b = _run(kw, ref=True)
    for k in a[3]:
        assert np.array_equal(a[3][k], b[3][k]), k
    for k in a[4]:
        assert np.array_equal(a[4][k], b[4][k]), k
    for fld in ("vx", "vz", "sxx"):
        assert np.array_equal(a[5].array("wave", fld), b[5].array("wave", fld)), fld


@pytest.mark.parametrize("nd,freesurf", [(2, 0), (2, 1), (3, 0), (3, 1)])
def test_boundary_shell_maps_are_inverse(nd, freesurf):
    """savebnd's gid -> cell and inject_ind's cell -> gid agree
    (src/savebnd*.cl vs src/header_injectbnd.cl)."""
    import ctypes as C

    from oracle.oracle import Oracle

    cfg, _, _ = make_case(nd=nd, freesurf=freesurf, nz=30, ny=26, nx=28, nab=6, nt=4)
    o = Oracle(cfg)
    seen = set()
    i, j, k = C.c_int(), C.c_int(), C.c_int()
    for gid in range(o.nbnd):
        # with a free surface NBND (Init_OpenCL.c:988-1021) counts more
        # slots than the shells hold; those slots stay unused
        if not o.lib.fdo_savebnd_cell(o.h, gid, C.byref(i), C.byref(j), C.byref(k)):
            continue
        assert o.lib.fdo_inject_ind(o.h, k.value, j.value, i.value) == gid
        seen.add((i.value, j.value, k.value))
    if freesurf:
        assert o.nbnd >= len(seen)
    else:
        assert o.nbnd == len(seen)
    # every cell inject_ind maps is a saved cell
    NX, NY, NZ = o.NXp, o.NYp, o.NZp
    count = 0
    for x in range(NX):
        for y in range(NY):
            for z in range(NZ):
                if o.lib.fdo_inject_ind(o.h, z, y, x) != -1:
                    count += 1
                    assert (x, y, z) in seen
    assert count == len(seen)


DFT_LIVE = [
    (dict(nd=2, freesurf=1, L=0, nt=120, seed=1), [10.0, 18.0, 25.0]),
    (dict(nd=2, freesurf=0, L=2, nt=120, seed=2), [10.0, 18.0, 25.0]),
    (dict(nd=3, freesurf=0, L=1, nz=30, ny=28, nx=32, nt=60, nab=6, seed=5, src_type=1), [20.0, 35.0]),
    (dict(nd=3, freesurf=1, L=0, nz=30, ny=28, nx=32, nt=60, nab=6, seed=6, src_type=2), [20.0, 35.0]),
]


@pytest.mark.skipif(not _ref_available(), reason="reference tree not present")
@pytest.mark.parametrize("param_type", [0, 1, 2])
@pytest.mark.parametrize("case", DFT_LIVE, ids=lambda c: "nd%d-L%d" % (c[0]["nd"], c[0]["L"]))
def test_dft_gradient_matches_reference_build(case, param_type):
    """BACK_PROP_TYPE=2 against the reference: the adjoint kernels compiled
    with BACK_PROP_TYPE=2 give the same transforms bit for bit; the oracle's
    calc_grad agrees with the reference's compiled calc_grad."""
    from oracle.oracle import ref_calc_grad
    from tests.golden.make_golden import DFT_NAMES

    kw, freqs = case
    extra = dict(back_prop_type=2, gradfreqs=freqs, param_type=param_type)
    got = []
    for ref in (False, True):
        from tests.golden.make_golden import model_inputs
        from oracle.oracle import Oracle

        cfg, model, acq = make_case(**kw)
        cfg.update(extra)
        o = Oracle(cfg, ref=ref)
        a, b, rho = model_inputs(model, param_type)
        assert o.set_model(a, b, rho, model["taup"], model["taus"]) == 0
        outs = ["vx", "vy", "vz"] if cfg["nd"] == 3 else ["vx", "vz"]
        d = o.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
        o.clear_gradients()
        o.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], {k: (0.3 * v).astype(np.float32) for k, v in d.items()})
        got.append((o, o.raw_gradients()))
    (o0, g0), (o1, g1) = got
    for slot in (0, 1):
        for n in DFT_NAMES:
            a = o0.dft(slot, "wave", n)
            if a is not None:
                assert np.array_equal(a, o1.dft(slot, "wave", n)), (slot, n)
    for k in g0:
        assert np.array_equal(g0[k], g1[k]), k
    gr = ref_calc_grad(o0)
    for k in gr:
        scale = np.abs(gr[k]).max()
        assert np.isfinite(g0[k]).all(), k
        assert np.abs(g0[k] - gr[k]).max() <= 1e-6 * scale, k


HESS_LIVE = [
    (dict(nd=2, freesurf=1, L=0, nt=120, seed=1), dict(hout=1)),
    (dict(nd=2, freesurf=0, L=0, nt=120, seed=2, abs_type=2), dict(hout=1, restype=1)),
    (dict(nd=2, freesurf=0, L=2, nt=120, seed=3), dict(hout=1)),
    (dict(nd=2, freesurf=1, L=0, nt=120, seed=4), dict(hout=1, back_prop_type=2, gradfreqs=[10.0, 18.0])),
    (dict(nd=2, freesurf=0, L=1, nt=120, seed=5), dict(hout=1, back_prop_type=2, gradfreqs=[10.0, 25.0])),
]


@pytest.mark.skipif(not _ref_available(), reason="reference tree not present")
@pytest.mark.parametrize("case", HESS_LIVE, ids=lambda c: "-".join("%s%s" % kv for kv in c[1].items() if kv[0] != "gradfreqs"))
def test_hessian_matches_reference_build(case):
    """Approximate Hessian (HOUT): the boundary-saving form bit for bit
    against the reference's 2D adjoint kernels compiled with HOUT=1; the DFT
    form against the reference's calc_grad compiled in place."""
    from oracle.oracle import Oracle, ref_calc_grad

    kw, extra = case
    got = []
    for ref in (False, True):
        cfg, model, acq = make_case(**kw)
        cfg.update(extra)
        o = Oracle(cfg, ref=ref)
        assert o.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"]) == 0
        d = o.forward(acq["src_pos"], acq["src"], acq["rec_pos"], ["vx", "vz"], save_boundaries=True)
        o.clear_gradients()
        o.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], {k: (0.3 * v).astype(np.float32) for k, v in d.items()})
        got.append((o, o.hessians(transform=False)))
    (o0, h0), (o1, h1) = got
    assert np.abs(h0["M"]).max() > 0
    for k in h0:
        assert np.array_equal(h0[k], h1[k]), k
    if extra.get("back_prop_type") == 2:
        r = ref_calc_grad(o0)
        for k in h0:
            scale = np.abs(r["H" + k]).max()
            assert np.abs(h0[k] - r["H" + k]).max() <= 1e-6 * scale, k
