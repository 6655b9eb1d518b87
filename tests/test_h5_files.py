"""The HDF5 job files and the command line (SeisCL's file protocol).

* seiscl_b200.h5lite round-trips what SeisCL writes (scalars and arrays of
  the csts, models, seismograms; empty arrays; more datasets than one
  symbol-table node holds), reads a chunked, deflate-compressed dataset (the
  layout of the reference's outputs, src/writehdf5.c:24-90), and reads a
  file written by the HDF5 library itself with a 512-byte user block (a
  MATLAB 7.3 file that ships with scipy's test data).
* The job under tests/golden/job_psv2d was written by the reference's own
  SeisCL class (tests/golden/make_job_files.py); the front end reads its
  constants back with the reference's transposes.
* ``python -m seiscl_b200.cli <base>`` fails with one line on stderr and a
  nonzero status when the job files are missing (no device needed), and
  (GPU) runs the reference-written job to the same seismograms, residuals,
  misfit and gradients as the in-memory path of the Python class.
"""
import json
import os
import shutil
import struct
import subprocess
import sys
import zlib

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JOB = os.path.join(ROOT, "tests", "golden", "job_psv2d")


def test_h5lite_round_trip(tmp_path):
    from seiscl_b200 import h5lite

    rng = np.random.default_rng(0)
    d = {"N": np.array([300, 400], np.int64), "dt": 1e-3, "NT": 2000, "FL": np.array([15.0, 30.0]),
         "vp": rng.random((40, 30)).astype(np.float32), "src_pos": rng.random((3, 5)),
         "i32": np.arange(7, dtype=np.int32), "u16": np.arange(5, dtype=np.uint16),
         "gradfreqs": np.empty((0, 1)), "vol": rng.random((4, 5, 6)).astype(np.float32)}
    for i in range(100):
        d["x%03d" % i] = np.float64(i)
    p = str(tmp_path / "f.mat")
    h5lite.write(p, d)
    back = h5lite.read(p)
    assert set(back) == set(d)
    for k, v in d.items():
        v = np.asarray(v)
        assert back[k].shape == v.shape and back[k].dtype == v.dtype, k
        assert np.array_equal(back[k], v), k


def _chunked_file(path, arr, chunk):
    """A file with one chunked, deflate-compressed float32 dataset "a"
    (layout message v3 class 2, filter pipeline v1, v1 B-tree of chunks),
    built by hand from the format specification."""
    from seiscl_b200 import h5lite as H

    UNDEF = H.UNDEF
    rank = arr.ndim
    chunks = []
    for i0 in range(0, arr.shape[0], chunk[0]):
        for i1 in range(0, arr.shape[1], chunk[1]):
            blk = np.zeros(chunk, np.float32)
            part = arr[i0:i0 + chunk[0], i1:i1 + chunk[1]]
            blk[:part.shape[0], :part.shape[1]] = part
            chunks.append(((i0, i1), zlib.compress(blk.tobytes(), 6)))
    out = bytearray(b"\x00" * 96)
    root_at = len(out)
    out += b"\x00" * len(H._ohdr_v1([H._msg(0x11, b"\x00" * 16)]))
    heap_at = len(out)
    out += b"HEAP" + struct.pack("<B3xQQQ", 0, 16, UNDEF, heap_at + 32) + b"\x00" * 8 + b"a\x00" + b"\x00" * 6
    snod_at = len(out)
    out += b"\x00" * (8 + 8 * 40)
    gtree_at = len(out)
    out += b"\x00" * (24 + 33 * 8 + 32 * 8)
    data_at = []
    for _, c in chunks:
        data_at.append(len(out))
        out += c + b"\x00" * (-len(c) % 8)
    ksz = 8 + 8 * (rank + 1)
    ctree_at = len(out)
    node = b"TREE" + struct.pack("<BBHQQ", 1, 0, len(chunks), UNDEF, UNDEF)
    for (off, c), at in zip(chunks, data_at):
        node += struct.pack("<II", len(c), 0) + b"".join(struct.pack("<Q", o) for o in off) + struct.pack("<Q", 0)
        node += struct.pack("<Q", at)
    node += struct.pack("<II", 0, 0) + b"".join(struct.pack("<Q", s) for s in arr.shape) + struct.pack("<Q", 0)
    out += node
    layout = struct.pack("<BBB", 3, 2, rank + 1) + struct.pack("<Q", ctree_at) + \
        b"".join(struct.pack("<I", c) for c in chunk) + struct.pack("<I", 4)
    pipeline = struct.pack("<BB6x", 1, 1) + struct.pack("<HHHH", 1, 8, 0, 1) + b"deflate\x00" + struct.pack("<I", 6) + \
        b"\x00" * 4
    ds_at = len(out)
    out += H._ohdr_v1([H._msg(0x01, H._space_msg(arr.shape)), H._msg(0x03, H._dtype_msg(np.dtype(np.float32))),
                       H._msg(0x0B, pipeline), H._msg(0x08, layout)])
    sb = H.SIGNATURE + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0, 4, 16, 0)
    sb += struct.pack("<QQQQ", 0, UNDEF, len(out), UNDEF)
    sb += struct.pack("<QQII", 0, root_at, 1, 0) + struct.pack("<QQ", gtree_at, heap_at)
    out[0:len(sb)] = sb
    r = H._ohdr_v1([H._msg(0x11, struct.pack("<QQ", gtree_at, heap_at))])
    out[root_at:root_at + len(r)] = r
    sn = b"SNOD" + struct.pack("<BBH", 1, 0, 1) + struct.pack("<QQII", 8, ds_at, 0, 0) + b"\x00" * 16
    out[snod_at:snod_at + len(sn)] = sn
    gt = b"TREE" + struct.pack("<BBHQQ", 0, 0, 1, UNDEF, UNDEF) + struct.pack("<QQQ", 0, snod_at, 8)
    out[gtree_at:gtree_at + len(gt)] = gt
    with open(path, "wb") as fh:
        fh.write(bytes(out))


def test_h5lite_reads_chunked_deflate(tmp_path):
    from seiscl_b200 import h5lite

    a = np.random.default_rng(1).standard_normal((19, 13)).astype(np.float32)
    p = str(tmp_path / "c.mat")
    _chunked_file(p, a, (19, 8))   # the reference's chunking: all of dim 0, 8 along dim 1
    got = h5lite.read(p)["a"]
    assert got.dtype == np.float32 and np.array_equal(got, a)


def test_h5lite_reads_a_library_written_file():
    """A MATLAB 7.3 file (written by the HDF5 library: 512-byte user block,
    base address 512, symbol-table root group, v1 object headers): the
    variable testdouble = 0:pi/4:2*pi."""
    import scipy

    from seiscl_b200 import h5lite

    p = os.path.join(os.path.dirname(scipy.__file__), "io", "matlab", "tests", "data", "testhdf5_7.4_GLNX86.mat")
    if not os.path.exists(p):
        pytest.skip("scipy's MATLAB 7.3 test file is not installed")
    d = h5lite.read(p)
    assert list(d) == ["testdouble"]
    assert np.allclose(d["testdouble"].ravel(), np.arange(9) * np.pi / 4)


def test_reference_written_constants_read_back():
    """The constants file written by the reference's SeisCL.write_csts is
    read by the front end with the reference's transposes."""
    from seiscl_b200.seiscl import SeisCL

    meta = json.load(open(os.path.join(JOB, "job.json")))
    s = SeisCL(file="SeisCL", workdir=JOB, files=True)
    s.read_csts()
    assert list(np.atleast_1d(s.N)) == meta["N"]
    assert s.NT == meta["NT"] and s.ND == meta["ND"] and s.nab == meta["nab"]
    assert abs(s.dt - meta["dt"]) < 1e-15 and s.gradout == 1 and s.rmsout == 1
    sp = np.asarray(meta["src_pos_all"])
    assert s.src_pos.shape == (5, sp.shape[1]) and np.array_equal(s.src_pos, sp)
    assert s.rec_pos.shape[0] == 8 and s.src.shape == (meta["NT"], sp.shape[1])


def test_cli_reports_missing_job_files(tmp_path):
    r = subprocess.run([sys.executable, "-m", "seiscl_b200.cli", str(tmp_path / "nothing")], cwd=ROOT,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode != 0
    assert "could not read parameter file" in r.stderr
    r = subprocess.run([sys.executable, "-m", "seiscl_b200.cli", "-z", "x"], cwd=ROOT, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode != 0 and "Unknown option" in r.stderr


@pytest.mark.gpu
def test_cli_job_matches_in_memory_path(tmp_path, cuda_device):
    """The reference-written job through the command line (files in, files
    out) and through the Python class in memory: identical seismograms,
    residuals, misfit and gradients."""
    from seiscl_b200.seiscl import SeisCL

    work = tmp_path / "job"
    shutil.copytree(JOB, work)
    r = subprocess.run([sys.executable, "-m", "seiscl_b200.cli", str(work / "SeisCL")], cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert r.stderr == ""
    for f in ("SeisCL_dout.mat", "SeisCL_gout.mat", "SeisCL_rms.mat"):
        assert (work / f).exists(), f
    files = SeisCL(file="SeisCL", workdir=str(work), files=True)
    files.read_csts()
    files.to_load_names = ["vx", "vz"]
    got = (files.read_data(), files.read_data(residuals=True), files.read_grad(), files.read_rms())

    meta = json.load(open(os.path.join(JOB, "job.json")))
    inp = np.load(os.path.join(JOB, "inputs.npz"))
    mem = SeisCL(N=np.array(meta["N"]), ND=meta["ND"], dh=meta["dh"], dt=meta["dt"], NT=meta["NT"],
                 nab=meta["nab"], freesurf=meta["freesurf"], L=meta["L"], f0=meta["f0"], FDORDER=meta["FDORDER"],
                 seisout=meta["seisout"], rmsout=meta["rmsout"], resout=meta["resout"], FL=np.array(15),
                 VPPML=3500, FPML=15, NPOWER=2, K_MAX_CPML=2, abpc=6)
    mem.src_pos_all = np.asarray(meta["src_pos_all"])
    mem.rec_pos_all = np.asarray(meta["rec_pos_all"])
    mem.src_all = np.asarray(meta["src_all"])
    mem.prepare_data(meta["srcids"])
    mem.write_data({"vx": inp["obs_vx"], "vz": inp["obs_vz"]})
    mem.set_forward(meta["srcids"], {k: inp[k] for k in ("vp", "vs", "rho")}, withgrad=True)
    mem.execute()
    mem.to_load_names = ["vx", "vz"]
    want = (mem.read_data(), mem.read_data(residuals=True), mem.read_grad(), mem.read_rms())
    for a, b in zip(got[0] + got[1] + got[2], want[0] + want[1] + want[2]):
        assert a.shape == b.shape
        assert np.abs(b).max() > 0
        assert np.array_equal(a, b)
    assert np.allclose(np.asarray(got[3][0]), np.asarray(want[3][0]), rtol=1e-6)
    assert np.allclose(np.asarray(got[3][1]), np.asarray(want[3][1]), rtol=1e-6)
