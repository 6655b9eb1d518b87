"""Analytical reference traces for tests/test_analytic.py, computed with the
REFERENCE'S own analytical modules (SeisCL/analytical: viscoelastic.py --
homogeneous 2D/3D (visco)elastic space, garvin2.py -- Garvin's 2D
half-space, lamb3D.py -- Lamb's 3D half-space), with the acquisitions,
source wavelets and resampling of SeisCL/tests/test_analytics.py:234-460.

The modules import matplotlib at the top (for plotting only); an empty
stand-in is registered so they load here.  Run from the repository root
(needs the reference tree):

    python tests/golden/make_analytic.py [/path/to/reference]

Output: tests/golden/analytic.npz -- for every case the normalised
analytical section (NT x ntraces, float32) and the acquisition the test
rebuilds the finite-difference run from.
"""
import importlib.util
import json
import os
import sys
import time
import types

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
OUT = os.path.join(ROOT, "tests", "golden", "analytic.npz")

# SeisCL/tests/test_analytics.py:53-96 (define_SeisCL) defaults
BASE = dict(dt=0.25e-3, NT=800, dh=2.0, f0=20.0, FDORDER=4, N=300, nab=112, abpc=3.0)


def ricker(f0, NT, dt):
    # test_analytics.py:33-50
    tmin = -1.5 / f0
    t = np.linspace(tmin, (NT - 1) * dt + tmin, num=NT)
    return (1.0 - 2.0 * (np.pi ** 2) * (f0 ** 2) * (t ** 2)) * np.exp(-(np.pi ** 2) * (f0 ** 2) * (t ** 2))


def load(ref_root, name):
    if "matplotlib" not in sys.modules:
        mpl = types.ModuleType("matplotlib")
        plt = types.ModuleType("matplotlib.pyplot")
        mpl.pyplot = plt
        sys.modules["matplotlib"] = mpl
        sys.modules["matplotlib.pyplot"] = plt
    spec = importlib.util.spec_from_file_location("ref_" + name, os.path.join(ref_root, "SeisCL", "analytical",
                                                                              name + ".py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def acquisition(kind, ND, testtype):
    """Source and receivers of test_analytics.py (cells of the N^ND grid)."""
    N, nab, dh, nbuf = BASE["N"], BASE["nab"], BASE["dh"], BASE["FDORDER"] * 2
    if kind == "lamb3d":                       # :234-300
        sx, sy, sz = (nab + nbuf) * dh, N // 2 * dh, 0.0
        offmin, offmax = 5 * dh, (N - nab - nbuf) * dh - sx
        gx = np.arange(sx + offmin, sx + offmax, dh)
        gy, gz = gx * 0 + sy, 0 * gx
        st = 0 if testtype == "inline" else 1
        return (sx, sy, sz, st), (gx, gy, gz, st), gx - sx
    if kind == "garvin2d":                     # :303-363
        sx, sy, sz = (nab + nbuf) * dh, 0.0, dh * 10
        offmin, offmax = 5 * dh, (N - nab - nbuf) * dh - sx
        gx = np.arange(sx + offmin, sx + offmax, dh)
        return (sx, sy, sz, 100), (gx, gx * 0, gx * 0 + dh * 10, 0), gx - sx + dh / 2
    # homogeneous space, :365-446
    if testtype == "inline":
        sx = sy = N // 2 * dh
        sz = (nab + nbuf) * dh
        offmin, offmax = 5 * dh, (N - nab - nbuf) * dh - sz
        gz = np.arange(sz + offmin, sz + offmax, dh)
        gx = gy = gz * 0 + N // 2 * dh
        off = gz - sz
    else:
        sx, sy, sz = (nab + nbuf) * dh, N // 2 * dh, N // 2 * dh
        offmin, offmax = 5 * dh, (N - nab - nbuf) * dh - sx
        gx = np.arange(sx + offmin, sx + offmax, dh)
        gy = gz = gx * 0 + N // 2 * dh
        off = gx - sx
    if ND == 2:
        sy, gy = 0.0, gy * 0
    return (sx, sy, sz, 2), (gx, gy, gz, 2), off


CASES = [
    # name, kind, ND, testtype, taup=taus, L
    ("lamb3d_inline", "lamb3d", 3, "inline", 0.0, 0),
    ("garvin2d", "garvin2d", 2, None, 0.0, 0),
    ("elastic3d_inline", "homog", 3, "inline", 0.0, 0),
    ("viscoelastic3d_crossline", "homog", 3, "crossline", 0.1, 1),
    ("elastic2d_crossline", "homog", 2, "crossline", 0.0, 0),
    ("viscoelastic2d_inline", "homog", 2, "inline", 0.2, 1),
]


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    ve, garvin2, lamb3d = load(ref_root, "viscoelastic"), load(ref_root, "garvin2"), load(ref_root, "lamb3D")
    vp, vs, rho = 3500.0, 2000.0, 2000.0
    NT, dt, f0 = BASE["NT"], BASE["dt"], BASE["f0"]
    out, meta = {}, {"base": BASE, "vp": vp, "vs": vs, "rho": rho, "cases": {}}
    for name, kind, ND, tt, tau, L in CASES:
        t0 = time.time()
        src, rec, off = acquisition(kind, ND, tt)
        FL = [f0 / (l + 1) for l in range(L)]
        if kind == "lamb3d":
            resamp = 500
            s = ricker(f0, resamp * NT - 1, dt / resamp)
            an = lamb3d.compute_shot(off, vp, vs, rho, dt / resamp, s, srctype="x", rectype="x", linedir="x")
            an = an[::resamp, :] / np.max(an[::resamp, :])
            norm = "max"
        elif kind == "garvin2d":
            resamp = 50
            s = ricker(f0, resamp * NT - 1, dt / resamp)
            an = garvin2.compute_shot(off, vp, vs, rho, dt / resamp, s, rectype="x", zsrc=src[2], zrec=rec[2][0])
            an = an[::resamp, :]
            an = an / np.sqrt(np.sum(an ** 2))
            norm = "l2"
        else:
            s = ricker(f0, 2 * NT, dt)
            gx, gy, gz, _ = rec
            rp = [[gx[i] - src[0], gy[i] - src[1], gz[i] - src[2]] for i in range(len(gx))]
            fn = ve.viscoelastic_3D if ND == 3 else ve.viscoelastic_2D
            an = fn(vp, vs, rho, tau, tau, f0, np.array(FL), dt, rp, s)[-1][:NT, :]
            an = an / np.sqrt(np.sum(an ** 2))
            norm = "l2"
        out[name] = np.asarray(an, np.float32)
        meta["cases"][name] = dict(kind=kind, ND=ND, testtype=tt, tau=tau, L=L, FL=FL, norm=norm,
                                   src=[float(v) for v in src], rec=[np.asarray(r).tolist() for r in rec[:3]],
                                   rectype=int(rec[3]), offsets=np.asarray(off).tolist())
        print(name, an.shape, "%.1f s" % (time.time() - t0))
    np.savez_compressed(OUT, meta=json.dumps(meta), **out)
    print("wrote", OUT, os.path.getsize(OUT))


if __name__ == "__main__":
    main()
