"""Generate the golden vectors in tests/golden/ from the reference's own
kernel sources, compiled in place (oracle/build.py:build_ref), driven by the
restated SeisCL time loop.

Run in a container where the reference tree is present:
    python tests/golden/make_golden.py [case ...]
(no names: every case).  The inputs are regenerated from seeds by
tests/_cases.make_case; a hash of them is stored beside the outputs so a
changed generator is caught.

The DFT-gradient cases (BACK_PROP_TYPE=2) run the reference's adjoint kernels
compiled with BACK_PROP_TYPE=2 and take the gradient from the reference's own
calc_grad (src/calc_grad.c compiled in place, oracle.oracle.ref_calc_grad);
the transforms are stored as float64 checksums (sum, sum of squares, max |.|).
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Oracle  # noqa: E402
from tests._cases import make_case  # noqa: E402

CASES = {
    "psv2d_fs_elastic": dict(nd=2, freesurf=1, L=0, abs_type=1, src_type=100),
    "psv2d_visco_l1": dict(nd=2, freesurf=0, L=1, abs_type=1, src_type=2),
    "psv2d_taper_fd4": dict(nd=2, freesurf=0, L=0, abs_type=2, src_type=100, fdorder=4),
    "el3d_fs_elastic": dict(nd=3, freesurf=1, L=0, abs_type=1, src_type=100, nz=36, ny=34, nx=38, nt=100, nab=8),
    "el3d_visco_l2": dict(nd=3, freesurf=1, L=2, abs_type=1, src_type=2, nz=36, ny=34, nx=38, nt=100, nab=8),
    "acoustic2d_l1": dict(nd=22, freesurf=0, L=1, abs_type=1, src_type=3),
    "sh2d_elastic": dict(nd=21, freesurf=0, L=0, abs_type=2, src_type=1),
}


# name: (make_case kwargs, extra configuration)
DFT_CASES = {
    "psv2d_dft_visco_l2": (dict(nd=2, freesurf=1, L=2, abs_type=1, src_type=100, nt=120, seed=11),
                           dict(back_prop_type=2, gradfreqs=[10.0, 18.0, 25.0], param_type=0)),
    "psv2d_dft_elastic_ip": (dict(nd=2, freesurf=0, L=0, abs_type=2, src_type=2, nt=120, seed=12),
                             dict(back_prop_type=2, gradfreqs=[12.0, 20.0], param_type=2)),
    "el3d_dft_visco_l1_m": (dict(nd=3, freesurf=1, L=1, abs_type=1, src_type=100, nz=30, ny=28, nx=32, nt=60,
                                 nab=6, seed=13),
                            dict(back_prop_type=2, gradfreqs=[20.0, 35.0], param_type=1)),
}
DFT_NAMES = ["vx", "vz", "sxx", "szz", "sxz", "vy", "syy", "sxy", "syz"]


def model_inputs(model, param_type):
    """vp/vs/rho converted to the parametrisation param_type expects."""
    vp, vs, rho = model["vp"], model["vs"], model["rho"]
    if param_type == 1:
        return (rho * vp * vp).astype(np.float32), (rho * vs * vs).astype(np.float32), rho
    if param_type == 2:
        return (rho * vp).astype(np.float32), (rho * vs).astype(np.float32), rho
    return vp, vs, rho


def checksum(a):
    v = np.asarray(a).view(np.float32).astype(np.float64)
    return np.array([v.sum(), (v * v).sum(), np.abs(v).max()])


def run_dft(kw, extra, ref=True):
    """Forward + DFT adjoint of one case.  Returns the inputs, seismograms,
    the gradient (the reference's calc_grad when ref=True, else the
    oracle's) and the checksums of the transforms."""
    from oracle.oracle import ref_calc_grad

    cfg, model, acq = make_case(**kw)
    cfg.update(extra)
    o = Oracle(cfg, ref=ref)
    a, b, rho = model_inputs(model, extra.get("param_type", 0))
    assert o.set_model(a, b, rho, model["taup"], model["taus"]) == 0
    outs = ["vx", "vy", "vz"] if cfg["nd"] == 3 else ["vx", "vz"]
    d = o.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
    o.clear_gradients()
    o.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], {k: (0.3 * v).astype(np.float32) for k, v in d.items()})
    g = ref_calc_grad(o) if ref else o.raw_gradients()
    sums = {}
    for slot in (0, 1):
        for n in DFT_NAMES:
            arr = o.dft(slot, "wave", n)
            if arr is not None:
                sums["dft%d_%s" % (slot, n)] = checksum(arr)
    return cfg, model, acq, d, g, sums


def input_hash(model, acq):
    h = hashlib.sha256()
    for d in (model, acq):
        for k in sorted(d):
            if d[k] is not None:
                h.update(k.encode())
                h.update(np.ascontiguousarray(d[k]).tobytes())
    return h.hexdigest()


def outputs_of(nd):
    return {3: ["vx", "vy", "vz", "p"], 21: ["vy", "sxy", "syz"]}.get(nd, ["vx", "vz", "p"])


def run(kw, ref=True):
    cfg, model, acq = make_case(**kw)
    o = Oracle(cfg, ref=ref)
    nd = cfg["nd"]
    rc = o.set_model(model["vp"] if nd != 21 else None, model["vs"] if nd != 22 else None, model["rho"],
                     model["taup"], model["taus"])
    assert rc == 0
    outs = outputs_of(nd)
    if nd in (21, 22):  # forward only in the reference
        return cfg, model, acq, o.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs), {}
    d = o.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs, save_boundaries=True)
    res = {k: (0.3 * v).astype(np.float32) for k, v in d.items() if k != "p"}
    o.clear_gradients()
    o.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], res)
    g = o.gradients()
    return cfg, model, acq, d, g


def main(names=None):
    path = os.path.join(HERE, "index.json")
    index = {}
    if names and os.path.exists(path):
        with open(path) as f:
            index = json.load(f)
    for name, (kw, extra) in DFT_CASES.items():
        if names and name not in names:
            continue
        cfg, model, acq, d, g, sums = run_dft(kw, extra, ref=True)
        out = {"seis_" + k: v for k, v in d.items()}
        out.update(sums)
        for k, v in g.items():
            if cfg["nd"] == 2:
                out["grad_" + k] = v
            else:
                out["gradsum_" + k] = checksum(v)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        index[name] = dict(kwargs=kw, extra=extra, input_sha256=input_hash(model, acq))
        print(name, "written")
    for name, kw in CASES.items():
        if names and name not in names:
            continue
        cfg, model, acq, d, g = run(kw, ref=True)
        out = {"seis_" + k: v for k, v in d.items()}
        if cfg["nd"] == 2:
            out.update({"grad_" + k: v for k, v in g.items()})
        else:
            for k, v in g.items():
                v64 = v.astype(np.float64)
                out["gradsum_" + k] = np.array([v64.sum(), (v64 * v64).sum(), np.abs(v64).max()])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        index[name] = dict(kwargs=kw, input_sha256=input_hash(model, acq))
        print(name, "written")
    with open(path, "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:] or None)
