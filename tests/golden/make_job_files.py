"""Write a SeisCL job (constants, model, observed data) with the REFERENCE'S
own Python class, for the file-protocol tests.

SeisCL/SeisCL.py writes its job files with h5py (write_csts, write_model,
write_data; SeisCL.py:658-763).  h5py, obspy and matplotlib are absent
here, so this script loads the reference module by path with stand-ins: an
``h5py`` whose ``File`` stores what the class assigns through
seiscl_b200.h5lite, and empty obspy/matplotlib modules (plotting and SEG-Y
are not used).  The constructor looks for a ``SeisCL_MPI`` executable on
PATH; a dummy one is put there.  Everything else -- which constants are
written, their types, the transposes, prepare_data's source/receiver
selection and receiver numbering -- is the reference's code.

Run from the repository root (needs the reference tree):

    python tests/golden/make_job_files.py [/path/to/reference]

Output: tests/golden/job_psv2d/{SeisCL_csts,SeisCL_model,SeisCL_din}.mat and
job.json (the parameters, for the tests).
"""
import importlib.util
import json
import os
import stat
import sys
import tempfile
import types

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
OUT = os.path.join(ROOT, "tests", "golden", "job_psv2d")


def _h5py_standin():
    from seiscl_b200 import h5lite

    class File:
        def __init__(self, path, mode="r"):
            self.path, self.mode = path, mode
            self.d = h5lite.read(path) if mode == "r" else {}

        def __enter__(self):
            return self

        def __exit__(self, *a):
            self.close()

        def close(self):
            if self.mode != "r":
                h5lite.write(self.path, self.d)

        def __setitem__(self, k, v):
            self.d[k.lstrip("/")] = np.asarray(v)

        def __getitem__(self, k):
            return self.d[k.lstrip("/")]

        def __contains__(self, k):
            return k.lstrip("/") in self.d

        def __iter__(self):
            return iter(self.d)

    return types.SimpleNamespace(File=File)


def _stub(name, **attrs):
    m = types.ModuleType(name)
    m.__dict__.update(attrs)
    sys.modules[name] = m
    return m


def load_reference_class(ref_root):
    sys.modules["h5py"] = _h5py_standin()
    _stub("obspy")
    _stub("obspy.core", Trace=object, Stream=object)
    _stub("obspy.io")
    _stub("obspy.io.segy")
    _stub("obspy.io.segy.segy", _read_segy=None)
    mpl = _stub("matplotlib", rcParams={})
    _stub("matplotlib.patches", Rectangle=object)
    _stub("matplotlib.pyplot")
    _stub("matplotlib.patheffects", withStroke=object)
    mpl.patches = sys.modules["matplotlib.patches"]
    spec = importlib.util.spec_from_file_location("ref_seiscl", os.path.join(ref_root, "SeisCL", "SeisCL.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


JOB = dict(N=[40, 50], ND=2, dh=10.0, dt=1e-3, NT=300, nab=10, freesurf=1, L=0, f0=15.0, FDORDER=8,
           seisout=1, rmsout=1, resout=1, gradout=1, srcids=[0, 1])


def model_and_data():
    rng = np.random.default_rng(7)
    nz, nx = JOB["N"]
    vp = (3000.0 * (1 + 0.03 * rng.standard_normal((nz, nx)))).astype(np.float32)
    vs = (vp / 1.8).astype(np.float32)
    rho = np.full((nz, nx), 2000.0, np.float32)
    return {"vp": vp, "vs": vs, "rho": rho}


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    mod = load_reference_class(ref_root)
    bindir = tempfile.mkdtemp()
    exe = os.path.join(bindir, "SeisCL_MPI")
    with open(exe, "w") as fh:
        fh.write("#!/bin/sh\nexit 0\n")
    os.chmod(exe, os.stat(exe).st_mode | stat.S_IEXEC)
    os.environ["PATH"] = bindir + os.pathsep + os.environ.get("PATH", "")
    j = JOB
    s = mod.SeisCL(N=np.array(j["N"]), ND=j["ND"], dh=j["dh"], dt=j["dt"], NT=j["NT"], nab=j["nab"],
                   freesurf=j["freesurf"], L=j["L"], f0=j["f0"], FDORDER=j["FDORDER"], seisout=j["seisout"],
                   rmsout=j["rmsout"], resout=j["resout"], workdir=OUT)
    s.surface_acquisition_2d(dg=3, ds=20, dsx=2, dsz=3, dgsz=3)
    os.makedirs(OUT, exist_ok=True)
    params = model_and_data()
    s.prepare_data(j["srcids"])
    ntr = s.rec_pos.shape[1]
    rng = np.random.default_rng(11)
    obs = {"vx": (1e-9 * rng.standard_normal((j["NT"], ntr))).astype(np.float32),
           "vz": (1e-9 * rng.standard_normal((j["NT"], ntr))).astype(np.float32)}
    s.write_data(dict(obs), workdir=OUT)
    s.set_forward(j["srcids"], params, workdir=OUT, withgrad=True)
    meta = dict(j)
    meta["src_pos_all"] = s.src_pos_all.tolist()
    meta["rec_pos_all"] = s.rec_pos_all.tolist()
    meta["src_all"] = np.asarray(s.src_all).tolist()
    with open(os.path.join(OUT, "job.json"), "w") as fh:
        json.dump(meta, fh)
    np.savez_compressed(os.path.join(OUT, "inputs.npz"), **params, **{"obs_" + k: v for k, v in obs.items()})
    print("wrote", sorted(os.listdir(OUT)))


if __name__ == "__main__":
    main()
