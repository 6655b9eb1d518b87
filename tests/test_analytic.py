"""Finite-difference seismograms against analytical solutions.

The analytical sections in tests/golden/analytic.npz were computed by the
reference's own analytical modules (SeisCL/analytical: Lamb's 3D
half-space, Garvin's 2D half-space, the homogeneous 2D/3D (visco)elastic
space) by tests/golden/make_analytic.py.  Each test reruns the matching
finite-difference modelling of SeisCL/tests/test_analytics.py:53-460
through the front end of this package -- 300-cell grids, dh = 2 m,
dt = 0.25 ms, 800 steps, 4th-order stencils, 112-cell Cerjan taper
(abpc 3), 20 Hz Ricker -- normalises both sections as the reference test
does and requires the reference's own bound: normalised RMSE <= 6e-2
(compare_data, test_analytics.py:142-165).
"""
import json
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = 6e-2


def _golden():
    d = np.load(os.path.join(ROOT, "tests", "golden", "analytic.npz"))
    return d, json.loads(str(d["meta"]))


def _cases():
    _, meta = _golden()
    return sorted(meta["cases"])


def fd_section(meta, name):
    """The finite-difference run of the case through SeisCL's front end
    (fd_solution, test_analytics.py:98-140)."""
    from seiscl_b200.seiscl import SeisCL

    b, c = meta["base"], meta["cases"][name]
    ND = c["ND"]
    seis = SeisCL()
    seis.ND = ND
    seis.N = np.array([b["N"]] * ND)
    seis.dt, seis.NT, seis.dh, seis.f0 = b["dt"], b["NT"], b["dh"], b["f0"]
    seis.L = c["L"]
    seis.FL = np.array(c["FL"]) if c["L"] else np.array([])
    seis.freesurf = 1 if c["kind"] in ("lamb3d", "garvin2d") else 0
    seis.FDORDER, seis.MAXRELERROR = b["FDORDER"], 1
    seis.abs_type, seis.seisout, seis.nab, seis.abpc = 2, 1, b["nab"], b["abpc"]
    sx, sy, sz, st = c["src"]
    seis.src_pos_all = np.stack([[sx], [sy], [sz], [0], [st]], axis=0)
    gx, gy, gz = (np.asarray(v) for v in c["rec"])
    seis.rec_pos_all = np.stack([gx, gy, gz, gz * 0, np.arange(len(gz)), gx * 0 + c["rectype"], gx * 0, gx * 0], 0)
    shape = tuple(seis.N)
    tau = c["tau"]
    params = {"vp": np.full(shape, meta["vp"]), "vs": np.full(shape, meta["vs"]), "rho": np.full(shape, meta["rho"]),
              "taup": np.full(shape, tau), "taus": np.full(shape, tau)}
    seis.set_forward(seis.src_pos_all[3, :], params, withgrad=False)
    seis.execute()
    data = seis.read_data()
    seis.close()
    return data[c["rectype"]] if c["kind"] in ("lamb3d", "garvin2d") else data[-1]


def rmse(fd, an, norm):
    fd = np.asarray(fd, np.float64)
    an = np.asarray(an, np.float64)
    if norm == "max":
        fd = fd / np.max(fd)
    else:
        fd = fd / np.sqrt(np.sum(fd ** 2))
    return float(np.sqrt(np.sum((fd - an) ** 2) / np.sum(an ** 2)))


def test_analytic_fixture_is_consistent():
    """The stored sections are normalised as the reference test normalises
    them and carry their acquisition (no device needed)."""
    d, meta = _golden()
    assert len(meta["cases"]) >= 6
    for name, c in meta["cases"].items():
        a = d[name].astype(np.float64)
        assert a.shape == (meta["base"]["NT"], len(c["offsets"]))
        if c["norm"] == "max":
            assert abs(a.max() - 1.0) < 1e-6
        else:
            assert abs(np.sum(a ** 2) - 1.0) < 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("name", _cases())
def test_fd_matches_analytic(name, cuda_device):
    d, meta = _golden()
    fd = fd_section(meta, name)
    err = rmse(fd, d[name], meta["cases"][name]["norm"])
    path = os.environ.get("SEISCL_PARITY_REPORT")
    if path:
        with open(path, "a") as fh:
            fh.write(json.dumps({"case": "analytic " + name, "normalised_rmse": err}) + "\n")
    assert err <= TOL, (name, err)
