"""Reference values of SeisCL's constant-Q fit for tests/test_qfit.py.

Loads the REFERENCE'S SeisCL/Q_tau.py by path (matplotlib, imported there
for plotting only, replaced by an empty stand-in) and records, for a few
calibrations, the relaxation frequencies after QTAU.tau_optimize() and
Q2tau at several Q.  Run from the repository root (needs the reference tree):

    python tests/golden/make_qtau.py [/path/to/reference]
"""
import importlib.util
import json
import os
import sys
import types

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
OUT = os.path.join(ROOT, "tests", "golden", "qtau.json")

CASES = [
    # qmin, qmax, fmin, fmax, initial FL, Q values
    (10.0, 200.0, 5.0, 40.0, "band2", [20.0, 50.0, 100.0]),
    (7.0, 200.0, 15.0, 80.0, [5.0, 30.0, 60.0], [7.0, 20.0, 50.0]),
    (20.0, 100.0, 2.0, 25.0, "band1", [30.0, 50.0]),
]


def load_qtau(ref_root):
    mpl = types.ModuleType("matplotlib")
    mpl.rcParams = {}
    mpl.pyplot = types.ModuleType("matplotlib.pyplot")
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", mpl.pyplot)
    spec = importlib.util.spec_from_file_location("ref_q_tau", os.path.join(ref_root, "SeisCL", "Q_tau.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def initial_fl(spec, fmin, fmax):
    from seiscl_b200.qfit import band_frequencies

    if isinstance(spec, str):
        return band_frequencies(int(spec[4:]), fmin, fmax)
    return list(spec)


def reference_values(m):
    out = []
    for qmin, qmax, fmin, fmax, fl0, qs in CASES:
        fl0 = initial_fl(fl0, fmin, fmax)
        q = m.QTAU(qmin, qmax, fmin, fmax, list(fl0))
        before = [float(q.Q2tau(v)) for v in qs]
        q.tau_optimize()
        out.append(dict(qmin=qmin, qmax=qmax, fmin=fmin, fmax=fmax, fl0=fl0, q=qs, tau_before=before,
                        fl=[float(v) for v in q.get_FL()], tau=[float(q.Q2tau(v)) for v in qs]))
    return out


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    vals = reference_values(load_qtau(ref))
    with open(OUT, "w") as fh:
        json.dump(vals, fh, indent=1)
    print("wrote", OUT)
