"""Generate the golden vectors in tests/golden/ from the reference's own
kernel sources, compiled in place (oracle/build.py:build_ref), driven by the
restated SeisCL time loop.

Run in a container where the reference tree is present:
    python tests/golden/make_golden.py
The inputs are regenerated from seeds by tests/_cases.make_case; a hash of
them is stored beside the outputs so a changed generator is caught.
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


def main():
    index = {}
    for name, kw in CASES.items():
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
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
