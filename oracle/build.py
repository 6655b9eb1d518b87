"""Build recipes for the CPU oracle.

TEST INFRASTRUCTURE ONLY: the checker of the CUDA path, never the product.

* ``build_port()`` compiles the C restatement (fdo_setup.c, fdo_port.c,
  fdo_driver.c) into ``oracle/_build/libfdo_port.so``.  It needs only gcc and
  runs anywhere, including the GPU box.
* ``build_ref_gpu(cfg, hc)`` compiles the reference's 3D forward CUDA
  kernels in place with nvcc for sm_100a (oracle/ref_gpu_tu.cu) into
  ``oracle/_ref/libfdo_refgpu_<key>.so``: the reference's own GPU code, for
  parity and timing beside this package's kernels (tests only).
* ``build_ref(cfg)`` compiles the reference's own kernel sources *in place*
  from the reference tree (``SEISCL_REF_SRC``, else ``reference/src`` beside
  the repository) with the same -D constants the reference passes at run time
  (src/clprogram.c:449-571), links them with ref_glue.c and the restated time
  loop, and writes ``oracle/_ref/libfdo_ref_<key>.so``.  Nothing from the
  reference tree is copied.  Each grid needs its own build because the
  reference fixes sizes at compile time.

The port and the pinning build of the reference use -O2 -ffp-contract=off so
the two agree bit for bit.  For timing the reference on the host cores
(the benchmark's CPU baseline and reference arm) ``build_ref(cfg, speed=...)``
makes two more builds of the same sources with ``-O3 -fopenmp`` and
``-march=x86-64-v3`` (AVX2 + FMA, any current x86-64 server) or
``-march=native`` (this build machine's instruction set, recorded beside the
library so a run on another CPU can tell whether it may load it).
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
REF_SRC = os.environ.get("SEISCL_REF_SRC",
                         os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference", "src"))
CFLAGS = ["-O2", "-fPIC", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-std=gnu17", "-w"]
SPEED_FLAGS = {"v3": ["-O3", "-march=x86-64-v3", "-fPIC", "-fopenmp", "-std=gnu17", "-w"],
               "native": ["-O3", "-march=native", "-fPIC", "-fopenmp", "-std=gnu17", "-w"]}
PORT_SOURCES = ["fdo_setup.c", "fdo_port.c", "fdo_driver.c", "fdo_dft.c"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed: %s\n%s" % (" ".join(cmd), r.stderr[-4000:]))


def port_lib_path(fp64: bool = False) -> str:
    return os.path.join(BUILD, "libfdo_port64.so" if fp64 else "libfdo_port.so")


def build_port(force: bool = False, fp64: bool = False) -> str:
    """The restatement as a shared library; fp64: its FP64 build (FDO_FP64)."""
    out = port_lib_path(fp64)
    srcs = [os.path.join(HERE, s) for s in PORT_SOURCES + ["fdo.h"]]
    if not force and os.path.exists(out):
        if os.path.getmtime(out) >= max(os.path.getmtime(s) for s in srcs):
            return out
    os.makedirs(BUILD, exist_ok=True)
    tmp = out + ".tmp%d" % os.getpid()
    _run(["gcc", *CFLAGS, *(["-DFDO_FP64"] if fp64 else []), "-shared", "-o", tmp,
          *[os.path.join(HERE, s) for s in PORT_SOURCES], "-lm"])
    os.replace(tmp, out)
    return out


def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_SRC, "update_v2D.cl"))


def _literal(v: float) -> str:
    return "%9.9f" % v


def ref_defines(cfg: dict, nbnd: int, hc: list) -> list:
    """The -D constants of src/clprogram.c:449-571 for a single device."""
    nd = cfg["nd"]
    F = cfg["fdorder"] // 2
    f32 = lambda x: float(ctypes.c_float(x).value)
    dt = f32(cfg["dt"])
    dh = f32(cfg["dh"])
    d = {
        "NZ": cfg["nz"] + 2 * F,
        "NX": cfg["nx"] + 2 * F,
        "FDOH": F,
        "NAB": cfg["nab"],
        "LVE": cfg.get("L", 0),
        "ND": nd,
        "NDIM": 3 if nd == 3 else 2,
        "ABS_TYPE": cfg.get("abs_type", 1),
        "FREESURF": cfg.get("freesurf", 0),
        "DT": _literal(dt),
        "DT2": _literal(dt / 2.0),
        "DH": _literal(dh),
        "DTDH": _literal(f32(dt / dh)),
        "NT": cfg["nt"],
        "OFFSET": 0,
        "DEVID": 0,
        "NUM_DEVICES": 1,
        "MYLOCALID": 0,
        "NLOCALP": 1,
        "LCOMM": 0,
        "COMM12": 0,
        "BACK_PROP_TYPE": cfg.get("back_prop_type", 1),
        "RESTYPE": cfg.get("restype", 0),
        "HOUT": cfg.get("hout", 0),
        "GRADSRCOUT": 0,
        "GRADOUT": 1,
        "FP16": 0,
        "NFREQS": 0,
        "NBND": nbnd,
        "NTNYQ": 0,
        "DTNYQ": 0,
    }
    if nd == 3:
        d["NY"] = cfg["ny"] + 2 * F
    for i in range(6):
        d["HC%d" % (i + 1)] = _literal(hc[i + 1])
    return ["-D%s=%s" % (k, v) for k, v in d.items()]


KERNELS = {
    2: [("update_v2D.cl", "update_v", 1, False), ("update_s2D.cl", "update_s", 1, False),
        ("surface2D.cl", "freesurface", 0, False), ("update_adjv2D.cl", "update_adjv", 1, True),
        ("update_adjs2D.cl", "update_adjs", 1, True), ("surface2D_adj.cl", "surface_adj", 0, False),
        ("savebnd2D.cl", "savebnd", 1, False)],
    3: [("update_v3D.cl", "update_v", 1, False), ("update_s3D.cl", "update_s", 1, False),
        ("surface3D.cl", "freesurface", 0, False), ("update_adjv3D.cl", "update_adjv", 1, True),
        ("update_adjs3D.cl", "update_adjs", 1, True), ("surface3D_adj.cl", "surface_adj", 0, False),
        ("savebnd3D.cl", "savebnd", 1, False)],
    # SH: the reference's stress kernel does not compile for L>0 and its
    # surface kernel cannot be loaded (named "surface"), so only v and s
    21: [("update_v2D_SH.cl", "update_v", 1, False), ("update_s2D_SH.cl", "update_s", 1, False)],
    # acoustic: forward only in the reference
    22: [("update_v2D_acc.cl", "update_v", 1, False), ("update_s2D_acc.cl", "update_s", 1, False)],
}


def ref_key(cfg: dict) -> str:
    keys = ["nd", "nz", "ny", "nx", "fdorder", "maxrelerror", "nab", "freesurf", "abs_type", "L", "nt",
            "dt", "dh", "restype", "back_prop_type", "hout"]
    blob = json.dumps({k: cfg.get(k) for k in keys}, sort_keys=True)
    return hashlib.sha1(blob.encode()).hexdigest()[:16]


def ref_lib_path(cfg: dict, speed: str = "pin") -> str:
    suffix = "" if speed == "pin" else "_" + speed
    return os.path.join(REF_OUT, "libfdo_ref_%s%s.so" % (ref_key(cfg), suffix))


def cpu_flags() -> set:
    """Instruction-set flags of this machine's CPU (/proc/cpuinfo)."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def native_usable(path: str) -> bool:
    """Whether a -march=native build may run here: every instruction-set flag
    of the machine that built it is present on this CPU."""
    try:
        built = set(json.load(open(path + ".cpu.json"))["flags"])
    except (OSError, ValueError, KeyError):
        return False
    return built <= cpu_flags()


def build_ref(cfg: dict, nbnd: int, hc: list, speed: str = "pin") -> str:
    """Compile the reference kernels for this grid (needs the reference tree).
    speed "pin": the bit-exact pinning build; "v3" / "native": -O3 timing
    builds (see the module docstring)."""
    out = ref_lib_path(cfg, speed)
    flags = CFLAGS if speed == "pin" else SPEED_FLAGS[speed]
    if os.path.exists(out):
        return out
    if not ref_available():
        raise FileNotFoundError("reference kernel sources not found at %s" % REF_SRC)
    os.makedirs(REF_OUT, exist_ok=True)
    nd = cfg["nd"]
    defs = ref_defines(cfg, nbnd, hc)
    with tempfile.TemporaryDirectory() as td:
        objs = []
        for fname, entry, local_off, inject in KERNELS[nd]:
            obj = os.path.join(td, entry + ".o")
            cmd = ["gcc", *flags, "-c", "-o", obj, os.path.join(HERE, "ref_tu.c"), "-I" + HERE,
                   "-I" + REF_SRC, *defs, "-DLOCAL_OFF=%d" % local_off,
                   "-DREF_KERNEL_FILE=%s" % fname, "-D%s=ref_%s" % (entry, entry)]
            if inject:
                cmd += ["-DREF_WITH_INJECT=1", "-Dinject_ind=inject_ind_%s" % entry]
            _run(cmd)
            objs.append(obj)
        glue = os.path.join(td, "glue.o")
        gdefs = [d for d in defs if d.split("=")[0] in ("-DND", "-DNX", "-DNY", "-DNZ", "-DFDOH")]
        _run(["gcc", *flags, "-c", "-o", glue, os.path.join(HERE, "ref_glue.c"), "-I" + HERE, *gdefs])
        tmp = out + ".tmp%d" % os.getpid()
        _run(["gcc", *flags, "-shared", "-o", tmp, glue, *objs,
              *[os.path.join(HERE, s) for s in PORT_SOURCES], "-lm"])
        if speed == "native":
            with open(out + ".cpu.json", "w") as fh:
                json.dump({"flags": sorted(cpu_flags())}, fh)
        os.replace(tmp, out)
    return out


NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
# the reference's 3D forward kernels, compiled for the GPU: file, entry point
GPU_KERNELS = [("update_v3D.cl", "update_v"), ("update_s3D.cl", "update_s"), ("surface3D.cl", "freesurface")]
GPU_BLOCK = (32, 4, 4)   # src/Init_OpenCL.c:493-500 for 3D: 32 x FDORDER/2 x FDORDER/2 at order 8


def ref_gpu_lib_path(cfg: dict) -> str:
    return os.path.join(REF_OUT, "libfdo_refgpu_%s.so" % ref_key(cfg))


def build_ref_gpu(cfg: dict, hc: list) -> str:
    """Compile the reference's 3D forward CUDA kernels (update_v3D.cl,
    update_s3D.cl, surface3D.cl) in place for sm_100a, as its CUDA build
    compiles them with NVRTC (src/clprogram.c:449-571: the grid and physics
    constants as -D options, LOCAL_OFF 0, cuda_fp16.h pre-included), one
    translation unit per file (oracle/ref_gpu_tu.cu), into
    oracle/_ref/libfdo_refgpu_<key>.so with a launcher per kernel.  Each
    grid needs its own build; the update kernels need nz a multiple of 32
    and ny, nx multiples of 4 (the launch covers the grid exactly)."""
    out = ref_gpu_lib_path(cfg)
    if os.path.exists(out):
        return out
    if cfg["nd"] != 3 or cfg["fdorder"] != 8:
        raise ValueError("the GPU build covers the 3D 8th-order kernels")
    if not ref_available():
        raise FileNotFoundError("reference kernel sources not found at %s" % REF_SRC)
    os.makedirs(REF_OUT, exist_ok=True)
    defs = ref_defines(cfg, 0, hc)
    arch = ["-gencode", "arch=compute_100a,code=sm_100a"]
    with tempfile.TemporaryDirectory() as td:
        objs = []
        for fname, entry in GPU_KERNELS:
            obj = os.path.join(td, entry + ".o")
            _run([NVCC, *arch, "-O3", "-std=c++17", "-w", "-Xcompiler", "-fPIC", "-c", "-o", obj,
                  os.path.join(HERE, "ref_gpu_tu.cu"), "-I" + HERE, "-I" + REF_SRC, *defs, "-DLOCAL_OFF=0",
                  "-DREF_KERNEL_FILE=%s" % fname, "-D%s=ref_gpu_%s" % (entry, entry),
                  "-DREF_ENTRY=ref_gpu_%s" % entry, "-DREF_LAUNCH=ref_gpu_launch_%s" % entry])
            objs.append(obj)
        tmp = out + ".tmp%d" % os.getpid()
        _run([NVCC, *arch, "-shared", "-o", tmp, *objs, "-lcudart"])
        os.replace(tmp, out)
    return out


def refcg_lib_path() -> str:
    return os.path.join(REF_OUT, "libfdo_refcg.so")


def build_refcg() -> str:
    """Compile the reference's host file src/calc_grad.c (the DFT-gradient
    assembly, OpenCL build) in place, with type-only stand-ins for the OpenCL
    and HDF5 headers (oracle/refstub) and a glue file that fills the
    reference's model/device structures (oracle/ref_calc_grad_glue.c)."""
    out = refcg_lib_path()
    if os.path.exists(out):
        return out
    if not ref_available():
        raise FileNotFoundError("reference sources not found at %s" % REF_SRC)
    os.makedirs(REF_OUT, exist_ok=True)
    flags = [*CFLAGS, "-D__SEISCL__", "-D__NOMPI__", "-I" + os.path.join(HERE, "refstub"), "-I" + REF_SRC]
    with tempfile.TemporaryDirectory() as td:
        o1 = os.path.join(td, "calc_grad.o")
        o2 = os.path.join(td, "glue.o")
        _run(["gcc", *flags, "-c", "-o", o1, os.path.join(REF_SRC, "calc_grad.c")])
        _run(["gcc", *flags, "-c", "-o", o2, os.path.join(HERE, "ref_calc_grad_glue.c")])
        tmp = out + ".tmp%d" % os.getpid()
        _run(["gcc", *CFLAGS, "-shared", "-o", tmp, o1, o2, "-lm"])
        os.replace(tmp, out)
    return out


if __name__ == "__main__":
    print(build_port(force=True))
