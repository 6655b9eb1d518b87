"""ctypes binding of the CPU oracle.

TEST INFRASTRUCTURE ONLY.  This is the checker of the CUDA product path: only
tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use it.

``Oracle(cfg)`` runs the C restatement (fdo_port.c); ``Oracle(cfg, ref=True)``
runs the reference's own kernel sources compiled in place (oracle/_ref), with
the same restated time loop; ``Oracle(cfg, fp64=True)`` runs the FP64 build of
the restatement (every float of it retyped double, fdo.h FDO_FP64): the
double-precision result that FP32 and FP16-storage runs are measured against.
Its inputs are the same FP32 values (configuration floats and arrays are
rounded to FP32 first) and its outputs are float64.  Inputs and outputs follow SeisCL's host
conventions: models are [nx][nz] (2D) or [nx][ny][nz] (3D) arrays with z
fastest; src_pos is [nsrc][5], rec_pos [nrec][8], src [nsrc][NT]; seismograms
are [nrec][NT] per recorded variable.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

OUT_NAMES = ["vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "syz", "sxz", "p"]
WAVE_IDS = {"vx": 0, "vy": 1, "vz": 2, "sxx": 3, "syy": 4, "szz": 5, "sxy": 6, "syz": 7, "sxz": 8}
MEM_IDS = {"rxx": 0, "ryy": 1, "rzz": 2, "rxy": 3, "ryz": 4, "rxz": 5}
PARAM_IDS = {"M": 0, "mu": 1, "rho": 2, "taup": 3, "taus": 4, "rip": 5, "rjp": 6, "rkp": 7, "muipkp": 8,
             "muipjp": 9, "mujpkp": 10, "tausipkp": 11, "tausipjp": 12, "tausjpkp": 13}
PSI_IDS = {n: i for i, n in enumerate(
    ["psi_vx_x", "psi_vy_x", "psi_vz_x", "psi_vx_y", "psi_vy_y", "psi_vz_y", "psi_vx_z", "psi_vy_z",
     "psi_vz_z", "psi_sxx_x", "psi_sxy_x", "psi_sxz_x", "psi_sxy_y", "psi_syy_y", "psi_syz_y",
     "psi_sxz_z", "psi_syz_z", "psi_szz_z"])}


def _cfg_class(real):
    class _Cfg(C.Structure):
        _fields_ = [("nd", C.c_int), ("nz", C.c_int), ("ny", C.c_int), ("nx", C.c_int),
                    ("fdorder", C.c_int), ("fdoh", C.c_int), ("maxrelerror", C.c_int),
                    ("nab", C.c_int), ("freesurf", C.c_int), ("abs_type", C.c_int), ("L", C.c_int),
                    ("nt", C.c_int), ("tmin", C.c_int), ("tmax", C.c_int),
                    ("dt", real), ("dh", real), ("f0", real), ("fl", real * 8),
                    ("vppml", real), ("fpml", real), ("npower", real),
                    ("k_max_cpml", real), ("abpc", real),
                    ("param_type", C.c_int), ("restype", C.c_int), ("back_prop_type", C.c_int),
                    ("nfreqs", C.c_int), ("gradfreqs", real * 16), ("hout", C.c_int)]
    return _Cfg


fdo_cfg = _cfg_class(C.c_float)
fdo_cfg64 = _cfg_class(C.c_double)     # the FDO_FP64 build's layout


DEFAULTS = dict(nd=2, ny=1, fdorder=8, maxrelerror=1, nab=16, freesurf=0, abs_type=1, L=0, tmin=0,
                tmax=0, f0=15.0, fl=(15.0,), vppml=3500.0, fpml=15.0, npower=2.0, k_max_cpml=2.0,
                abpc=6.0, param_type=0, restype=0, back_prop_type=1, gradfreqs=())


def make_cfg(cfg: dict, fp64: bool = False):
    d = dict(DEFAULTS)
    d.update(cfg)
    c = fdo_cfg64() if fp64 else fdo_cfg()
    for k in ["nd", "nz", "ny", "nx", "fdorder", "maxrelerror", "nab", "freesurf", "abs_type", "L", "nt",
              "tmin", "tmax", "param_type", "restype"]:
        setattr(c, k, int(d[k]))
    c.fdoh = int(d["fdorder"]) // 2
    if c.nd != 3:
        c.ny = 1
    for k in ["dt", "dh", "f0", "vppml", "fpml", "npower", "k_max_cpml", "abpc"]:
        setattr(c, k, float(np.float32(d[k])))
    fl = list(np.atleast_1d(d["fl"]).astype(np.float32).astype(float))
    for i in range(8):
        c.fl[i] = fl[i] if i < len(fl) else 0.0
    c.back_prop_type = int(d.get("back_prop_type", 1))
    gf = [float(v) for v in np.atleast_1d(d.get("gradfreqs", ())).ravel()]
    if len(gf) > 16:
        raise ValueError("at most 16 DFT gradient frequencies")
    c.nfreqs = len(gf)
    for i, v in enumerate(gf):
        c.gradfreqs[i] = float(np.float32(v))
    c.hout = int(d.get("hout", 0))
    return c


def _lib(path, real=C.c_float):
    lib = C.CDLL(path)
    P = C.c_void_p
    FP = C.POINTER(real)
    lib.fdo_create.restype = P
    lib.fdo_create.argtypes = [C.POINTER(fdo_cfg64 if real is C.c_double else fdo_cfg), C.c_int,
                               C.POINTER(C.c_int)]
    lib.fdo_destroy.argtypes = [P]
    lib.fdo_model.argtypes = [P, FP, FP, FP, FP, FP]
    lib.fdo_run_forward.argtypes = [P, C.c_int, FP, FP, C.c_int, FP, C.POINTER(C.c_int), C.c_int,
                                    C.POINTER(FP), C.c_int]
    lib.fdo_run_adjoint.argtypes = [P, C.c_int, FP, FP, C.c_int, FP, C.POINTER(C.c_int), C.c_int,
                                    C.POINTER(FP)]
    lib.fdo_get_grad.argtypes = [P, FP, FP, FP, FP, FP, FP]
    lib.fdo_get_grad_raw.argtypes = [P, C.POINTER(FP)]
    lib.fdo_get_hess.argtypes = [P, C.c_int, C.POINTER(FP)]
    lib.fdo_dft_array.restype = FP
    lib.fdo_dft_array.argtypes = [P, C.c_int, C.c_int, C.c_int]
    lib.fdo_dft_info.argtypes = [P, C.POINTER(C.c_int), FP, FP]
    lib.fdo_run_calc_grad.argtypes = [P]
    lib.fdo_clear_grad.argtypes = [P]
    lib.fdo_array.restype = FP
    lib.fdo_array.argtypes = [P, C.c_int, C.c_int]
    lib.fdo_info.argtypes = [P, C.POINTER(C.c_int64)]
    lib.fdo_run_steps.argtypes = [P, C.c_int]
    lib.fdo_holberg.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
    lib.fdo_source_targets.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), FP]
    lib.fdo_inject_ind.argtypes = [P, C.c_int, C.c_int, C.c_int]
    lib.fdo_savebnd_cell.argtypes = [P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    return lib


_PORT = None
_PORT64 = None


def port_lib():
    global _PORT
    if _PORT is None:
        _PORT = _lib(_build.build_port())
    return _PORT


def port_lib64():
    global _PORT64
    if _PORT64 is None:
        _PORT64 = _lib(_build.build_port(fp64=True), C.c_double)
    return _PORT64


def _fptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double if a.dtype == np.float64 else C.c_float))


def source_type_mask(src_pos: np.ndarray) -> int:
    """Bit t for source types 0..3 and bit 4 for type 100, over all shots
    (the reference scans every source of the acquisition,
    src/automatic_kernels.c:416-437)."""
    m = 0
    for t in np.asarray(src_pos).reshape(-1, 5)[:, 4].astype(np.int32):
        if 0 <= t < 4:
            m |= 1 << int(t)
        if t == 100:
            m |= 1 << 4
    return m


class Oracle:
    def __init__(self, cfg: dict, ref: bool = False, fp64: bool = False, speed: str = "pin"):
        if ref and fp64:
            raise ValueError("the reference kernels are FP32 only")
        self.cfg = dict(DEFAULTS)
        self.cfg.update(cfg)
        if self.cfg["nd"] != 3:
            self.cfg["ny"] = 1
        self.fp64 = fp64
        self.dtype = np.float64 if fp64 else np.float32
        self.real = C.c_double if fp64 else C.c_float
        self._c = make_cfg(self.cfg, fp64)
        self.lib = port_lib64() if fp64 else port_lib()
        if ref:
            h0 = self._make(self.lib, False)
            info = self._info(self.lib, h0)
            self.lib.fdo_destroy(h0)
            hc = (C.c_double * 7)()
            self.lib.fdo_holberg(self._c.fdorder, self._c.maxrelerror, hc)
            path = _build.build_ref(self.cfg, int(info[5]), list(hc), speed)
            self.lib = _lib(path)
        self.h = self._make(self.lib, ref)
        self.info = self._info(self.lib, self.h)
        self.NZp, self.NYp, self.NXp, self.nvol, self.npar, self.nbnd = [int(v) for v in self.info]

    def _make(self, lib, ref):
        err = C.c_int(0)
        h = lib.fdo_create(C.byref(self._c), 1 if ref else 0, C.byref(err))
        if err.value != 0:
            lib.fdo_destroy(h)
            raise RuntimeError("oracle init failed (%d)" % err.value)
        return h

    @staticmethod
    def _info(lib, h):
        out = (C.c_int64 * 6)()
        lib.fdo_info(h, out)
        return list(out)

    def close(self):
        if getattr(self, "h", None):
            self.lib.fdo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        c = self.cfg
        return (c["nx"], c["ny"], c["nz"]) if c["nd"] == 3 else (c["nx"], c["nz"])

    def set_model(self, vp, vs, rho, taup=None, taus=None) -> int:
        arrs = [None if a is None else
                np.ascontiguousarray(np.asarray(a, np.float32), dtype=self.dtype).reshape(self.shape)
                for a in (vp, vs, rho, taup, taus)]
        self._keep = arrs
        return self.lib.fdo_model(self.h, *[_fptr(a) for a in arrs])

    def _outsel(self, outputs):
        sel = (C.c_int * 10)()
        for n in outputs:
            sel[OUT_NAMES.index(n)] = 1
        return sel

    def _in(self, a):
        """An input array as the build takes it: FP32 values, in its type."""
        return np.ascontiguousarray(np.asarray(a, np.float32), dtype=self.dtype)

    def forward(self, src_pos, src, rec_pos, outputs, mask=None, save_boundaries=False):
        src_pos = self._in(src_pos).reshape(-1, 5)
        rec_pos = self._in(rec_pos).reshape(-1, 8)
        nt = self.cfg["nt"]
        src = self._in(src).reshape(src_pos.shape[0], nt)
        if mask is None:
            mask = source_type_mask(src_pos)
        nrec = rec_pos.shape[0]
        outs = {n: np.zeros((nrec, nt), self.dtype) for n in outputs}
        ptrs = (C.POINTER(self.real) * 10)()
        for n, a in outs.items():
            ptrs[OUT_NAMES.index(n)] = _fptr(a)
        rc = self.lib.fdo_run_forward(self.h, src_pos.shape[0], _fptr(src_pos), _fptr(src), nrec,
                                      _fptr(rec_pos), self._outsel(outputs), mask, ptrs,
                                      1 if save_boundaries else 0)
        if rc:
            raise RuntimeError("oracle forward failed (%d)" % rc)
        return outs

    def adjoint(self, src_pos, src, rec_pos, residuals: dict, mask=None):
        src_pos = self._in(src_pos).reshape(-1, 5)
        rec_pos = self._in(rec_pos).reshape(-1, 8)
        nt = self.cfg["nt"]
        src = self._in(src).reshape(src_pos.shape[0], nt)
        if mask is None:
            mask = source_type_mask(src_pos)
        res = {n: np.ascontiguousarray(r, self.dtype).reshape(rec_pos.shape[0], nt) for n, r in residuals.items()}
        ptrs = (C.POINTER(self.real) * 10)()
        for n, a in res.items():
            ptrs[OUT_NAMES.index(n)] = _fptr(a)
        rc = self.lib.fdo_run_adjoint(self.h, src_pos.shape[0], _fptr(src_pos), _fptr(src), rec_pos.shape[0],
                                      _fptr(rec_pos), self._outsel(list(res)), mask, ptrs)
        if rc:
            raise RuntimeError("oracle adjoint failed (%d)" % rc)

    def gradients(self):
        n = self.npar
        g = [np.zeros(n, self.dtype) for _ in range(6)]
        self.lib.fdo_get_grad(self.h, *[_fptr(a) for a in g])
        sh = self.shape
        return {"vp": g[0].reshape(sh), "vs": g[1].reshape(sh), "rho": g[2].reshape(sh),
                "rawM": g[3].reshape(sh), "rawmu": g[4].reshape(sh), "rawrho": g[5].reshape(sh)}

    def clear_gradients(self):
        self.lib.fdo_clear_grad(self.h)

    def raw_gradients(self) -> dict:
        """The float accumulators as they are (no transf_grad): M, mu, rho,
        taup, taus.  For the DFT gradient these are already in the
        param_type basis (calc_grad.c applies the chain rule itself)."""
        g = [np.zeros(self.npar, self.dtype) for _ in range(5)]
        ptrs = (C.POINTER(self.real) * 5)(*[_fptr(a) for a in g])
        self.lib.fdo_get_grad_raw(self.h, ptrs)
        sh = self.shape
        return {"rho": g[0].reshape(sh), "M": g[1].reshape(sh), "mu": g[2].reshape(sh),
                "taup": g[3].reshape(sh), "taus": g[4].reshape(sh)}

    def hessians(self, transform=True) -> dict:
        """Approximate Hessian (HOUT).  transform: the chain rule of
        transf_grad applied to the Hessian (src/calc_grad.c:1023-1060, no
        division by dt), keyed by the param_type's names; else the raw
        accumulators M, mu, rho, taup, taus."""
        g = [np.zeros(self.npar, self.dtype) for _ in range(5)]
        ptrs = (C.POINTER(self.real) * 5)(*[_fptr(a) for a in g])
        self.lib.fdo_get_hess(self.h, 1 if transform else 0, ptrs)
        sh = self.shape
        if transform:
            names = {0: ("vp", "vs"), 1: ("M", "mu"), 2: ("Ip", "Is")}[int(self.cfg.get("param_type", 0))]
            return {names[0]: g[1].reshape(sh), names[1]: g[2].reshape(sh), "rho": g[0].reshape(sh),
                    "taup": g[3].reshape(sh), "taus": g[4].reshape(sh)}
        return {"rho": g[0].reshape(sh), "M": g[1].reshape(sh), "mu": g[2].reshape(sh),
                "taup": g[3].reshape(sh), "taus": g[4].reshape(sh)}

    def dft_info(self) -> dict:
        """DTNYQ, NTNYQ, df and gradfreqsn of a DFT-gradient state
        (src/assign_modeling_case.c:549-570)."""
        ni = (C.c_int * 2)()
        df = self.real(0)
        fn = np.zeros(16, self.dtype)
        self.lib.fdo_dft_info(self.h, ni, C.byref(df), _fptr(fn))
        nf = len(np.atleast_1d(self.cfg.get("gradfreqs", ())))
        return {"dtnyq": ni[0], "ntnyq": ni[1], "df": df.value, "gradfreqsn": fn[:nf].copy()}

    def dft(self, slot: int, kind: str, name: str):
        """View (not a copy) of the complex DFT of a wave field ("wave") or a
        memory variable ("mem"): [nfreqs][(L)][nvol] complex64, slot 0
        forward, 1 adjoint; None when absent."""
        k, i = (0, WAVE_IDS[name]) if kind == "wave" else (1, MEM_IDS[name])
        p = self.lib.fdo_dft_array(self.h, slot, k, i)
        if not p:
            return None
        nf = len(np.atleast_1d(self.cfg.get("gradfreqs", ())))
        n = nf * self.nvol * (self.cfg["L"] if kind == "mem" else 1)
        return np.ctypeslib.as_array(p, shape=(2 * int(n),)).view(np.complex128 if self.fp64 else np.complex64)

    def calc_grad(self):
        """Assemble the DFT gradient from the transforms now held."""
        self.lib.fdo_run_calc_grad(self.h)

    def array(self, kind: str, name: str) -> np.ndarray:
        """Copy of an internal array (for field-level comparisons)."""
        a = self._view(kind, name)
        return None if a is None else a.copy()

    def set_array(self, kind: str, name: str, values) -> None:
        """Overwrite an internal array (a state to step from)."""
        a = self._view(kind, name)
        if a is None:
            raise KeyError("%s %s is not allocated" % (kind, name))
        a[:] = np.asarray(values, a.dtype).ravel()

    def _view(self, kind: str, name: str):
        c = self.cfg
        nab = c["nab"]
        if kind in ("wave", "adj"):
            k, i, n = (0 if kind == "wave" else 1), WAVE_IDS[name], self.nvol
        elif kind in ("mem", "adjmem"):
            k, i, n = (2 if kind == "mem" else 3), MEM_IDS[name], self.nvol * c["L"]
        elif kind == "psi":
            k, i = 4, PSI_IDS[name]
            ny = c["ny"]
            axis = name[-1]
            n = {"x": 2 * nab * ny * c["nz"], "y": c["nx"] * 2 * nab * c["nz"], "z": c["nx"] * ny * 2 * nab}[axis]
        elif kind == "param":
            k, i, n = 5, PARAM_IDS[name], self.npar
        elif kind in ("cpml_x", "cpml_y", "cpml_z"):
            k = {"cpml_x": 6, "cpml_y": 7, "cpml_z": 8}[kind]
            i = ["K", "a", "b", "K_half", "a_half", "b_half"].index(name)
            n = 2 * nab
        elif kind == "taper":
            k, i, n = 9, 0, nab
        elif kind == "eta":
            k, i, n = 10, 0, c["L"]
        elif kind == "bnd":
            k, i, n = 11, WAVE_IDS[name], self.nbnd * c["nt"]
        else:
            raise KeyError(kind)
        p = self.lib.fdo_array(self.h, k, i)
        if not p:
            return None
        return np.ctypeslib.as_array(p, shape=(int(n),))

    def residual_scale(self, rec_pos, residuals: dict) -> dict:
        """Adjoint-source scaling of src/residuals.c:452-568 (res_scale,
        FP16=0): velocity residuals times dt / (b * dh / dt) with b the
        buoyancy (rip/rjp/rkp) of the receiver's cell, whose x, y and z are
        all taken from rec_pos column 0 (residuals.c:487-489); pressure
        residuals times -2 (M - mu) dh / dt * dt, with the reference's mix of
        FP32 and double intermediates."""
        c = self.cfg
        rec_pos = np.ascontiguousarray(rec_pos, np.float32).reshape(-1, 8)
        nt = c["nt"]
        tmax = c.get("tmax", 0) or nt
        dh = np.float32(c["dh"])
        dt = np.float32(c["dt"])
        nz, ny = c["nz"], c["ny"]
        out = {}
        for name, r in residuals.items():
            r = np.array(r, dtype=np.float32, copy=True).reshape(rec_pos.shape[0], nt)
            if name in ("vx", "vy", "vz"):
                par = self.array("param", {"vx": "rip", "vy": "rjp", "vz": "rkp"}[name])
            elif name == "p":
                M = self.array("param", "M")
                mu = self.array("param", "mu")
            else:
                out[name] = r
                continue
            for g in range(rec_pos.shape[0]):
                if name == "p":
                    x, y, z = (int(rec_pos[g, k] / dh) for k in range(3))
                else:
                    x = y = z = int(rec_pos[g, 0] / dh)
                pos = (x * ny + y) * nz + z if c["nd"] == 3 else x * nz + z
                if name == "p":
                    # FP32 difference, double product, FP32 factor parscal*dt
                    parscal = np.float32(-2.0 * float(M[pos] - mu[pos]) * float(dh) / float(dt))
                    r[g, :tmax] *= np.float32(parscal * dt)
                else:
                    parscal = np.float32(1.0 / float(par[pos]) * float(dh) / float(dt))
                    f = 1.0 / float(parscal) * float(dt)
                    r[g, :tmax] = (r[g, :tmax].astype(np.float64) * f).astype(np.float32)
            out[name] = r
        return out

    def run_steps(self, n):
        self.lib.fdo_run_steps(self.h, n)


def holberg(fdorder: int, maxrelerror: int):
    hc = (C.c_double * 7)()
    if port_lib().fdo_holberg(fdorder, maxrelerror, hc):
        raise ValueError("bad FD order / error level")
    return list(hc)


DFT_VARS = ["vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "syz", "sxz", "rxx", "ryy", "rzz", "rxy", "ryz", "rxz"]


def ref_calc_grad(o: Oracle, fwd=None, adj=None) -> dict:
    """The reference's own calc_grad (src/calc_grad.c compiled in place,
    oracle/_ref) applied to copies of the transforms that `o` holds (or to
    the given {name: complex array} dicts), starting from zero gradients.
    Returns M, mu, rho, taup, taus as the reference's float host arrays."""
    lib = C.CDLL(_build.build_refcg())
    FP = C.POINTER(C.c_float)
    lib.refcg_run.argtypes = [C.c_int] * 10 + [C.c_float, C.c_float, FP, FP] + [C.POINTER(FP)] * 5
    c = o.cfg
    keep = []

    def buf(slot, given, name):
        if given is not None:
            a = given.get(name)
        else:
            a = o.dft(slot, "wave" if name in WAVE_IDS else "mem", name)
        if a is None:
            return None
        a = np.array(a, np.complex64, copy=True)
        keep.append(a)
        return a.view(np.float32).ctypes.data_as(FP)

    fw = (FP * 15)(*[buf(0, fwd, n) for n in DFT_VARS])
    ad = (FP * 15)(*[buf(1, adj, n) for n in DFT_VARS])
    L = int(c["L"])
    pars = [o.array("param", k) for k in ("M", "mu", "rho", "taup", "taus")]
    grads = [np.zeros(o.npar, np.float32) for _ in range(5)]
    hess = [np.zeros(o.npar, np.float32) for _ in range(5)]
    pp = (FP * 5)(*[_fptr(p) for p in pars])
    gp = (FP * 5)(*[_fptr(g) for g in grads])
    hp = (FP * 5)(*[_fptr(g) for g in hess]) if c.get("hout") else None
    info = o.dft_info()
    fl = np.zeros(8, np.float32)
    fl[:L] = np.atleast_1d(c["fl"])[:L]
    fn = np.ascontiguousarray(info["gradfreqsn"], np.float32)
    rc = lib.refcg_run(c["nd"], c["nz"], c["ny"], c["nx"], c["fdorder"], L, int(c["param_type"]), len(fn),
                       info["ntnyq"], info["dtnyq"], float(c["dt"]), float(c["f0"]), _fptr(fl), _fptr(fn), fw, ad, pp,
                       gp, hp)
    if rc:
        raise RuntimeError("reference calc_grad failed (%d)" % rc)
    sh = o.shape
    out = {k: g.reshape(sh) for k, g in zip(("M", "mu", "rho", "taup", "taus"), grads)}
    if c.get("hout"):
        out.update({"H" + k: g.reshape(sh) for k, g in zip(("M", "mu", "rho", "taup", "taus"), hess)})
    return out
