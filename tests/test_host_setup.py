"""Host-side set-up of the product (libseiscl_b200.so, no GPU needed) against
the oracle: parameter transforms, CPML profiles, source/receiver cells and
source targets.  Index work is bit-exact; FP64-computed coefficients agree
with the reference's FP32 computation to a few ulp (rtol 2e-6)."""
import numpy as np
import pytest

from tests._cases import engine_config, make_case

RTOL = 2e-6


@pytest.mark.parametrize("kw", [dict(nd=2, L=0), dict(nd=2, L=2, freesurf=0), dict(nd=3, L=2, nz=20, ny=18, nx=22, nab=4),
                                dict(nd=3, L=0, nz=20, ny=18, nx=22, nab=4)])
def test_transforms_match_oracle(kw):
    from oracle.oracle import Oracle
    from seiscl_b200 import engine

    cfg, model, _ = make_case(**kw)
    ours = engine.host_transform(engine_config(cfg), model["vp"], model["vs"], model["rho"], model["taup"],
                                 model["taus"])
    o = Oracle(cfg)
    assert o.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"]) == 0
    names = ["M", "mu", "rho", "rip", "rkp", "muipkp"]
    if cfg["nd"] == 3:
        names += ["rjp", "muipjp", "mujpkp"]
    if cfg["L"]:
        names += ["taup", "taus", "tausipkp"] + (["tausipjp", "tausjpkp"] if cfg["nd"] == 3 else [])
    for n in names:
        ref = o.array("param", n).reshape(ours[n].shape)
        np.testing.assert_allclose(ours[n], ref, rtol=RTOL, atol=0, err_msg=n)
        # the reference leaves some edge cells of the two-direction averages at zero
        assert np.array_equal(ours[n] == 0, ref == 0), n


def test_cpml_profiles_match_oracle():
    from oracle.oracle import Oracle
    from seiscl_b200 import engine

    cfg, _, _ = make_case(nd=2, nab=12)
    ours = engine.host_cpml(engine_config(cfg))
    o = Oracle(cfg)
    for i, n in enumerate(["K", "a", "b", "K_half", "a_half", "b_half"]):
        np.testing.assert_allclose(ours[i], o.array("cpml_x", n), rtol=RTOL, atol=1e-12, err_msg=n)


def test_point_cells_bit_exact():
    """(int)(pos/DH)+FDOH with the reference's DH literal, over awkward
    positions (negatives, exact multiples, dh that is not exact in binary)."""
    from seiscl_b200 import engine

    rng = np.random.default_rng(7)
    for dh in (10.0, 12.5, 0.1, 3.3, 7.77):
        cfg, _, _ = make_case(nd=3, nz=40, ny=30, nx=50, dh=dh)
        ec = engine_config(cfg)
        pos = np.zeros((400, 8), np.float32)
        pos[:, 0] = rng.uniform(-2 * dh, 52 * dh, 400)
        pos[:200, 0] = np.round(pos[:200, 0] / dh) * np.float32(dh)
        pos[:, 1] = rng.uniform(0, 29 * dh, 400)
        pos[:, 2] = rng.uniform(0, 39 * dh, 400)
        cells = engine.host_point_cells(ec, pos, 8)
        DH = float("%9.9f" % np.float32(dh))
        F = 4
        NZ, NY, NX = 48, 38, 58
        for r in range(400):
            i = int(float(pos[r, 0]) / DH) + F
            j = int(float(pos[r, 1]) / DH) + F
            k = int(float(pos[r, 2]) / DH) + F
            want = -1 if (i < F or i > NX - F - 1) else (i * NY + j) * NZ + k
            assert cells[r] == want, (dh, r, pos[r, :3])


@pytest.mark.parametrize("nd", [2, 3, 21, 22])
def test_source_targets_match_oracle(nd):
    import ctypes as C

    from oracle.oracle import port_lib
    from seiscl_b200 import engine

    lib = port_lib()
    names = ["vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "syz", "sxz"]
    for mask in range(1, 32):
        for stype in (0, 1, 2, 3, 100, 7):
            f = (C.c_int * 9)()
            d = (C.c_float * 9)()
            n = lib.fdo_source_targets(nd, mask, stype, f, d)
            ref = [(names[f[i]], float(d[i])) for i in range(n)]
            assert engine.host_source_targets(nd, mask, stype) == ref, (nd, mask, stype)
