"""ctypes binding of libseiscl_b200.so (the C ABI in include/seiscl_b200.h).

The product path: every call goes to the CUDA library.  There is no CPU
fallback; if the library cannot be loaded, or no CUDA device is present,
the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libseiscl_b200.so")

OUT_NAMES = ["vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "syz", "sxz", "p"]
PREC = {"fp32": 0, "fp16": 1, "bf16": 2}
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "CFL violated", -4: "out of device memory",
          -5: "call out of order", -6: "unstable", -7: "unsupported"}


class SeisCLEngineError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "error"), code, msg))
        self.code = code


class sfd_config(C.Structure):
    _fields_ = [("nd", C.c_int), ("n", C.c_int * 3), ("nt", C.c_int), ("fdorder", C.c_int),
                ("maxrelerror", C.c_int), ("L", C.c_int), ("freesurf", C.c_int), ("abs_type", C.c_int),
                ("nab", C.c_int), ("dt", C.c_float), ("dh", C.c_float), ("f0", C.c_float),
                ("fl", C.c_float * 8), ("vppml", C.c_float), ("fpml", C.c_float), ("npower", C.c_float),
                ("k_max_cpml", C.c_float), ("abpc", C.c_float), ("tmin", C.c_int), ("tmax", C.c_int),
                ("param_type", C.c_int), ("restype", C.c_int), ("precision", C.c_int),
                ("kernels", C.c_int), ("adjoint_reset_psi", C.c_int), ("field_precision", C.c_int),
                ("back_prop_type", C.c_int), ("loop_graphs", C.c_int), ("hout", C.c_int),
                ("batch", C.c_int), ("checkpoint", C.c_int)]


class sfd_shot(C.Structure):
    _fields_ = [("nsrc", C.c_int), ("nrec", C.c_int), ("src_pos", C.POINTER(C.c_float)),
                ("src", C.POINTER(C.c_float)), ("rec_pos", C.POINTER(C.c_float))]


FP = C.POINTER(C.c_float)
EXPORTS = {
    "sfd_plan_create": (C.c_int, [C.POINTER(sfd_config), C.POINTER(C.c_void_p)]),
    "sfd_plan_destroy": (None, [C.c_void_p]),
    "sfd_last_error": (C.c_char_p, [C.c_void_p]),
    "sfd_set_model": (C.c_int, [C.c_void_p, C.POINTER(FP)]),
    "sfd_source_type_mask": (C.c_int, [FP, C.c_int]),
    "sfd_forward": (C.c_int, [C.c_void_p, C.POINTER(sfd_shot), C.c_int, C.POINTER(C.c_int), C.POINTER(FP),
                              C.c_int, C.c_void_p]),
    "sfd_adjoint": (C.c_int, [C.c_void_p, C.POINTER(sfd_shot), C.c_int, C.POINTER(C.c_int), C.POINTER(FP),
                              C.c_void_p]),
    "sfd_forward_batch": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(sfd_shot), C.c_int, C.POINTER(C.c_int),
                                    C.POINTER(FP), C.c_int, C.c_void_p]),
    "sfd_adjoint_batch": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(sfd_shot), C.c_int, C.POINTER(C.c_int),
                                    C.POINTER(FP), C.c_void_p]),
    "sfd_zero_gradient": (C.c_int, [C.c_void_p]),
    "sfd_get_gradient": (C.c_int, [C.c_void_p, C.c_int, FP, FP, FP]),
    "sfd_get_gradient_q": (C.c_int, [C.c_void_p, FP, FP]),
    "sfd_get_hessian": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(FP)]),
    "sfd_set_gradfreqs": (C.c_int, [C.c_void_p, FP, C.c_int, C.POINTER(C.c_int)]),
    "sfd_set_movie": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(FP)]),
    "sfd_residual_scale": (C.c_int, [C.c_void_p, C.POINTER(sfd_shot), C.POINTER(C.c_int), C.POINTER(FP)]),
    "sfd_plan_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "sfd_plan_uses_tma": (C.c_int, [C.c_void_p]),
    "sfd_plan_kernel_family": (C.c_int, [C.c_void_p]),
    "sfd_plan_fused_step": (C.c_int, [C.c_void_p]),
    "sfd_debug_copy": (C.c_int64, [C.c_void_p, C.c_int, C.c_int, FP, C.c_int64]),
    "sfd_debug_load": (C.c_int64, [C.c_void_p, C.c_int, C.c_int, FP, C.c_int64]),
    "sfd_debug_launch": (C.c_int, [C.c_void_p, C.c_int]),
    "sfd_last_loop_ms": (C.c_float, [C.c_void_p]),
    "sfd_bench_kernels": (C.c_int, [C.c_void_p, C.c_int, FP]),
    "sfd_host_transform": (C.c_int, [C.POINTER(sfd_config), C.POINTER(FP), C.POINTER(FP)]),
    "sfd_host_point_cells": (C.c_int, [C.POINTER(sfd_config), FP, C.c_int, C.c_int, C.POINTER(C.c_int64)]),
    "sfd_host_source_targets": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_float)]),
    "sfd_host_cpml": (C.c_int, [C.POINTER(sfd_config), FP]),
    "sfd_footprint": (C.c_int, [C.POINTER(sfd_config), C.c_int, C.c_int, C.c_int64, C.c_int,
                                C.POINTER(C.c_int64)]),
    "sfd_device_memory": (C.c_int, [C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "sfd_plan_device_bytes": (C.c_int64, [C.c_void_p]),
    "sfd_release_memory": (C.c_int, []),
}

_LIB = None


def load_library(path: str = LIB_PATH):
    """Load the CUDA library.  Raises if it is missing: there is no fallback."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise FileNotFoundError("libseiscl_b200.so not built (run __graft_entry__.build()): %s" % path)
    lib = C.CDLL(path)
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None:
        a = a.reshape(shape)
    return a


def _ptr(a):
    return None if a is None else a.ctypes.data_as(FP)


def source_type_mask(src_pos) -> int:
    sp = _f32(src_pos).reshape(-1, 5)
    return int(load_library().sfd_source_type_mask(_ptr(sp), sp.shape[0]))


@dataclass
class Config:
    """The csts keys of SeisCL.py:23-30 used by the single-device path.

    ``N`` is [NZ, NX] (2D) or [NZ, NY, NX] (3D) as in SeisCL."""
    N: Sequence[int]
    ND: int = 2
    dh: float = 10.0
    dt: float = 0.0008
    NT: int = 875
    L: int = 0
    f0: float = 15.0
    FL: Sequence[float] = (15.0,)
    FDORDER: int = 8
    MAXRELERROR: int = 1
    freesurf: int = 0
    abs_type: int = 1
    VPPML: float = 3500.0
    NPOWER: float = 2.0
    FPML: float = 15.0
    K_MAX_CPML: float = 2.0
    nab: int = 16
    abpc: float = 6.0
    tmin: int = 0
    tmax: int = 0
    param_type: int = 0
    restype: int = 0
    precision: str = "fp32"
    kernels: str = "fast"  # "fast" (3D: 4-cell vectorised where eligible, else streaming), "general",
    #                        "register", "tma", "stream", "vector", "fused" ("fast" plus the fused
    #                        one-launch modelling step)
    adjoint_reset_psi: bool = False  # True: the adjoint starts from zeroed CPML memory (not the reference's)
    field_precision: str = "fp32"  # "fp16": wave fields / memory variables stored in FP16 (3D, 2D P-SV;
    #                                forward modelling and checkpointed gradients); "fp16_mem": memory
    #                                variables alone in FP16 (3D viscoelastic forward modelling)
    back_prop_type: int = 1  # 1: boundary-saving backpropagation, 2: DFT gradient at `gradfreqs`
    gradfreqs: Sequence[float] = ()  # DFT gradient frequencies (Hz), back_prop_type 2
    loop_graphs: str = "auto"  # time loops as CUDA graphs: "auto" (from the 2nd run of a loop), "always", "never"
    hout: int = 0  # HOUT: also accumulate the approximate Hessian (2D)
    batch: int = 1  # shots advanced together by forward_batch / adjoint_batch
    checkpoint: int = 0  # gradients: 0 boundary saving + backpropagation; K > 0 snapshots every K steps + recompute

    def to_c(self) -> sfd_config:
        c = sfd_config()
        c.nd = int(self.ND)
        n = list(self.N)
        for i in range(3):
            c.n[i] = int(n[i]) if i < len(n) else 0
        c.nt = int(self.NT)
        c.fdorder = int(self.FDORDER)
        c.maxrelerror = int(self.MAXRELERROR)
        c.L = int(self.L)
        c.freesurf = int(self.freesurf)
        c.abs_type = int(self.abs_type)
        c.nab = int(self.nab)
        c.dt = float(self.dt)
        c.dh = float(self.dh)
        c.f0 = float(self.f0)
        fl = list(np.atleast_1d(self.FL).astype(float))
        for i in range(8):
            c.fl[i] = fl[i] if i < len(fl) else 0.0
        c.vppml = float(self.VPPML)
        c.fpml = float(self.FPML)
        c.npower = float(self.NPOWER)
        c.k_max_cpml = float(self.K_MAX_CPML)
        c.abpc = float(self.abpc)
        c.tmin = int(self.tmin)
        c.tmax = int(self.tmax)
        c.param_type = int(self.param_type)
        c.restype = int(self.restype)
        c.precision = PREC[self.precision]
        c.kernels = {"fast": 0, "general": 1, "register": 2, "tma": 3, "stream": 4, "vector": 5,
                     "fused": 6, "async": 7}[self.kernels]
        c.adjoint_reset_psi = 1 if self.adjoint_reset_psi else 0
        c.batch = int(self.batch)
        c.checkpoint = int(self.checkpoint)
        c.field_precision = {"fp32": 0, "fp16": 1, "fp16_mem": 2}[self.field_precision]
        c.back_prop_type = int(self.back_prop_type)
        c.loop_graphs = {"auto": 0, "always": 1, "never": 2}[self.loop_graphs]
        c.hout = int(self.hout)
        return c

    @property
    def model_shape(self):
        """Host layout of a parameter array: [nx][nz] or [nx][ny][nz]."""
        n = list(self.N)
        return (n[2], n[1], n[0]) if self.ND == 3 else (n[1], n[0])


class Plan:
    """One grid on the current CUDA device (a thin wrapper of sfd_plan)."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        self.lib = load_library()
        self._c = cfg.to_c()
        h = C.c_void_p()
        rc = self.lib.sfd_plan_create(C.byref(self._c), C.byref(h))
        if rc:
            raise SeisCLEngineError(rc, "sfd_plan_create rejected the configuration")
        self.h = h
        info = (C.c_int64 * 8)()
        self.lib.sfd_plan_info(self.h, info)
        self.NZp, self.NYp, self.NXp, self.nvol, self.npar, self.nbnd, self.F, self.tmax = [int(v) for v in info]
        self.dtnyq = self.ntnyq = None
        if int(cfg.back_prop_type) == 2 and len(np.atleast_1d(cfg.gradfreqs)):
            self.set_gradfreqs(cfg.gradfreqs)

    def set_movie(self, movout: int, outputs=()):
        """Film `outputs` (wave-field names) every `movout` steps in the next
        runs (MOVOUT); returns {name: array [NT//movout][nx][(ny)][nz]} that
        those runs fill.  movout <= 0 turns it off."""
        self._movie = {}
        ptrs = (FP * 10)()
        if movout > 0:
            nslot = int(self.cfg.NT) // int(movout)
            for n in outputs:
                self._movie[n] = np.zeros((nslot,) + tuple(self.cfg.model_shape), np.float32)
                ptrs[OUT_NAMES.index(n)] = _ptr(self._movie[n])
        self._check(self.lib.sfd_set_movie(self.h, int(movout), ptrs))
        return self._movie

    def set_gradfreqs(self, freqs):
        """DFT-gradient frequencies (Hz); returns (DTNYQ, NTNYQ)."""
        f = _f32(np.atleast_1d(freqs)).ravel()
        info = (C.c_int * 2)()
        self._check(self.lib.sfd_set_gradfreqs(self.h, _ptr(f), int(f.size), info))
        self.nfreqs = int(f.size)
        self.dtnyq, self.ntnyq = int(info[0]), int(info[1])
        return self.dtnyq, self.ntnyq

    def _check(self, rc):
        if rc:
            raise SeisCLEngineError(rc, self.lib.sfd_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.sfd_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_model(self, vp, vs, rho, taup=None, taus=None):
        """Parameters in host layout [nx][(ny)][nz], z fastest."""
        sh = self.cfg.model_shape
        arrs = [None if a is None else _f32(a, sh) for a in (vp, vs, rho, taup, taus)]
        ptrs = (FP * 5)(*[_ptr(a) for a in arrs])
        self._check(self.lib.sfd_set_model(self.h, ptrs))

    @staticmethod
    def _shot(src_pos, src, rec_pos, nt):
        sp = _f32(src_pos).reshape(-1, 5)
        rp = _f32(rec_pos).reshape(-1, 8)
        s = _f32(src).reshape(sp.shape[0], nt)
        shot = sfd_shot(sp.shape[0], rp.shape[0], _ptr(sp), _ptr(s), _ptr(rp))
        return shot, (sp, s, rp)

    def forward(self, src_pos, src, rec_pos, outputs, mask=None, save_boundaries=False) -> Dict[str, np.ndarray]:
        nt = self.cfg.NT
        shot, keep = self._shot(src_pos, src, rec_pos, nt)
        if mask is None:
            mask = source_type_mask(src_pos)
        sel = (C.c_int * 10)()
        outs = {}
        ptrs = (FP * 10)()
        for n in outputs:
            i = OUT_NAMES.index(n)
            sel[i] = 1
            outs[n] = np.zeros((shot.nrec, nt), np.float32)
            ptrs[i] = _ptr(outs[n])
        self._check(self.lib.sfd_forward(self.h, C.byref(shot), int(mask), sel, ptrs,
                                         1 if save_boundaries else 0, None))
        return outs

    def adjoint(self, src_pos, src, rec_pos, residuals: Dict[str, np.ndarray], mask=None):
        nt = self.cfg.NT
        shot, keep = self._shot(src_pos, src, rec_pos, nt)
        if mask is None:
            mask = source_type_mask(src_pos)
        sel = (C.c_int * 10)()
        ptrs = (FP * 10)()
        res = {}
        for n, r in residuals.items():
            i = OUT_NAMES.index(n)
            sel[i] = 1
            res[n] = _f32(r, (shot.nrec, nt))
            ptrs[i] = _ptr(res[n])
        self._check(self.lib.sfd_adjoint(self.h, C.byref(shot), int(mask), sel, ptrs, None))

    def forward_batch(self, shots, outputs, mask=None, save_boundaries=False) -> List[Dict[str, np.ndarray]]:
        """Up to ``cfg.batch`` shots [(src_pos, src, rec_pos), ...] advanced
        together (one launch per kernel and step for all of them); returns
        their seismograms, one dict per shot."""
        nt = self.cfg.NT
        made = [self._shot(sp, src, rp, nt) for sp, src, rp in shots]
        arr = (sfd_shot * len(made))(*[m[0] for m in made])
        if mask is None:
            mask = source_type_mask(np.concatenate([m[1][0] for m in made]))
        nrec = [m[0].nrec for m in made]
        sel = (C.c_int * 10)()
        ptrs = (FP * 10)()
        flat = {}
        for n in outputs:
            i = OUT_NAMES.index(n)
            sel[i] = 1
            flat[n] = np.zeros((sum(nrec), nt), np.float32)
            ptrs[i] = _ptr(flat[n])
        self._check(self.lib.sfd_forward_batch(self.h, len(made), arr, int(mask), sel, ptrs,
                                               1 if save_boundaries else 0, None))
        cuts = np.cumsum([0] + nrec)
        return [{n: flat[n][cuts[b]:cuts[b + 1]] for n in outputs} for b in range(len(made))]

    def adjoint_batch(self, shots, residuals: Sequence[Dict[str, np.ndarray]], mask=None):
        """The adjoint of the batch a ``forward_batch(..., save_boundaries=True)``
        ran; ``residuals`` one dict per shot."""
        nt = self.cfg.NT
        made = [self._shot(sp, src, rp, nt) for sp, src, rp in shots]
        arr = (sfd_shot * len(made))(*[m[0] for m in made])
        if mask is None:
            mask = source_type_mask(np.concatenate([m[1][0] for m in made]))
        sel = (C.c_int * 10)()
        ptrs = (FP * 10)()
        flat = {}
        for n in residuals[0]:
            i = OUT_NAMES.index(n)
            sel[i] = 1
            flat[n] = np.ascontiguousarray(np.concatenate(
                [_f32(r[n], (m[0].nrec, nt)) for r, m in zip(residuals, made)]), np.float32)
            ptrs[i] = _ptr(flat[n])
        self._check(self.lib.sfd_adjoint_batch(self.h, len(made), arr, int(mask), sel, ptrs, None))

    def residual_scale(self, rec_pos, residuals: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
        nt = self.cfg.NT
        rp = _f32(rec_pos).reshape(-1, 8)
        shot = sfd_shot(0, rp.shape[0], None, None, _ptr(rp))
        sel = (C.c_int * 10)()
        ptrs = (FP * 10)()
        out = {}
        for n, r in residuals.items():
            i = OUT_NAMES.index(n)
            sel[i] = 1
            out[n] = np.array(r, dtype=np.float32, copy=True).reshape(rp.shape[0], nt)
            ptrs[i] = _ptr(out[n])
        self._check(self.lib.sfd_residual_scale(self.h, C.byref(shot), sel, ptrs))
        return out

    def zero_gradient(self):
        self._check(self.lib.sfd_zero_gradient(self.h))

    def gradient(self, transform=True):
        """Accumulated gradient.  Boundary-saving plans: of the param_type's
        parameters (transform=True) or of the stored M, mu, rho.  DFT plans:
        always of the param_type's parameters, plus taup and taus when L > 0."""
        sh = self.cfg.model_shape
        g = [np.zeros(sh, np.float32) for _ in range(3)]
        self._check(self.lib.sfd_get_gradient(self.h, 1 if transform else 0, *[_ptr(a) for a in g]))
        dft = int(self.cfg.back_prop_type) == 2
        if transform or dft:
            names = {0: ("vp", "vs", "rho"), 1: ("M", "mu", "rho"), 2: ("Ip", "Is", "rho")}[self.cfg.param_type]
        else:
            names = ("M", "mu", "rho")
        out = dict(zip(names, g))
        if dft and int(self.cfg.L) > 0:
            q = [np.zeros(sh, np.float32) for _ in range(2)]
            self._check(self.lib.sfd_get_gradient_q(self.h, *[_ptr(a) for a in q]))
            out["taup"], out["taus"] = q
        return out

    def hessian(self, transform=True):
        """Approximate Hessian (plans with hout=1), keyed as gradient()."""
        sh = self.cfg.model_shape
        h = [np.zeros(sh, np.float32) for _ in range(5)]
        self._check(self.lib.sfd_get_hessian(self.h, 1 if transform else 0, (FP * 5)(*[_ptr(a) for a in h])))
        dft = int(self.cfg.back_prop_type) == 2
        if transform or dft:
            names = {0: ("vp", "vs", "rho"), 1: ("M", "mu", "rho"), 2: ("Ip", "Is", "rho")}[self.cfg.param_type]
        else:
            names = ("M", "mu", "rho")
        out = dict(zip(names, h[:3]))
        if int(self.cfg.L) > 0:
            out["taup"], out["taus"] = h[3], h[4]
        return out

    def dft(self, slot: int, kind: str, name: str) -> np.ndarray:
        """Device transform (copy) of a wave field ("wave") or memory
        variable ("mem"), slot 0 forward / 1 adjoint, as complex64
        [nfreqs][(L)][padded cells]."""
        if kind == "wave":
            k, i, n = 6 + slot, OUT_NAMES.index(name), self.nvol
        else:
            k, i, n = 8 + slot, ["rxx", "ryy", "rzz", "rxy", "ryz", "rxz"].index(name), self.nvol * int(self.cfg.L)
        return self.debug_array(k, i, 2 * self.nfreqs * n).view(np.complex64)

    def debug_load(self, kind: int, idx: int, values) -> None:
        """Overwrite a device array (0 wave field, 1 adjoint wave field, 2
        memory variables) with ``values`` (tests)."""
        a = _f32(values).ravel()
        got = self.lib.sfd_debug_load(self.h, kind, idx, _ptr(a), a.size)
        if got < 0:
            self._check(int(got))

    def debug_launch(self, which: int) -> None:
        """Run one kernel on the plan's arrays: 0 velocity update, 1 stress
        update, 2 free surface, 3 free-surface adjoint (tests)."""
        self._check(self.lib.sfd_debug_launch(self.h, int(which)))

    def debug_array(self, kind: int, idx: int, n: int) -> np.ndarray:
        out = np.zeros(n, np.float32)
        got = self.lib.sfd_debug_copy(self.h, kind, idx, _ptr(out), n)
        if got < 0:
            self._check(int(got))
        return out[:got]

    def bench_kernels(self, nrep: int = 20):
        """Mean ms per launch of the (velocity, stress, surface, fused step)
        kernels; 0 for one the plan does not have."""
        out = (C.c_float * 4)()
        self._check(self.lib.sfd_bench_kernels(self.h, int(nrep), out))
        return list(out)

    @property
    def fused_step(self) -> bool:
        """True when 3D modelling runs advance each step in one fused launch
        (velocity, stress, memory variables, free surface)."""
        rc = int(self.lib.sfd_plan_fused_step(self.h))
        if rc < 0:
            self._check(rc)
        return rc == 1

    @property
    def uses_tma(self) -> bool:
        """True when the 3D stress update of this plan runs on the TMA-pipelined kernels."""
        rc = int(self.lib.sfd_plan_uses_tma(self.h))
        if rc < 0:
            self._check(rc)
        return rc == 1

    @property
    def device_bytes(self) -> int:
        """Device memory the plan holds now."""
        return int(self.lib.sfd_plan_device_bytes(self.h))

    @property
    def kernel_family(self) -> str:
        """Kernel family of the 3D stress update ("general", "register",
        "tma", "stream", "vector"; "2d" for 2D plans)."""
        rc = int(self.lib.sfd_plan_kernel_family(self.h))
        if rc < 0:
            self._check(rc)
        return ["2d", "general", "register", "tma", "stream", "vector"][rc]

    @property
    def last_loop_ms(self) -> float:
        return float(self.lib.sfd_last_loop_ms(self.h))


# ---------------------------------------------------------------- host-only
PARAM_NAMES = ["M", "mu", "rho", "taup", "taus", "rip", "rjp", "rkp", "muipkp", "muipjp", "mujpkp",
               "tausipkp", "tausipjp", "tausjpkp"]


def host_transform(cfg: Config, vp, vs, rho, taup=None, taus=None) -> Dict[str, np.ndarray]:
    """Transformed parameters exactly as sfd_set_model uploads them."""
    lib = load_library()
    sh = cfg.model_shape
    arrs = [None if a is None else _f32(a, sh) for a in (vp, vs, rho, taup, taus)]
    outs = [np.zeros(sh, np.float32) for _ in PARAM_NAMES]
    c = cfg.to_c()
    rc = lib.sfd_host_transform(C.byref(c), (FP * 5)(*[_ptr(a) for a in arrs]), (FP * 14)(*[_ptr(o) for o in outs]))
    if rc:
        raise SeisCLEngineError(rc, "host transform failed")
    return dict(zip(PARAM_NAMES, outs))


def host_point_cells(cfg: Config, pos, stride: int) -> np.ndarray:
    lib = load_library()
    p = _f32(pos).reshape(-1, stride)
    cells = np.zeros(p.shape[0], np.int64)
    c = cfg.to_c()
    rc = lib.sfd_host_point_cells(C.byref(c), _ptr(p), p.shape[0], stride, cells.ctypes.data_as(C.POINTER(C.c_int64)))
    if rc < 0:
        raise SeisCLEngineError(rc, "point mapping failed")
    return cells


def host_source_targets(nd: int, mask: int, stype: int):
    lib = load_library()
    f = (C.c_int * 3)()
    d = (C.c_float * 3)()
    n = lib.sfd_host_source_targets(nd, mask, stype, f, d)
    return [(OUT_NAMES[f[i]], float(d[i])) for i in range(n)]


def host_cpml(cfg: Config) -> np.ndarray:
    lib = load_library()
    out = np.zeros((6, 2 * cfg.nab), np.float32)
    c = cfg.to_c()
    rc = lib.sfd_host_cpml(C.byref(c), _ptr(out))
    if rc:
        raise SeisCLEngineError(rc, "cpml failed")
    return out


def footprint(cfg: Config, gradient: bool = False, nsrc: int = 1, nrec_sel: int = 0, nfreqs: int = 0) -> int:
    """Device bytes a plan for ``cfg`` allocates for shots of up to ``nsrc``
    sources and ``nrec_sel`` receiver traces (receivers x outputs), with a
    gradient run's buffers when ``gradient`` (no device call)."""
    lib = load_library()
    out = C.c_int64(0)
    rc = lib.sfd_footprint(C.byref(cfg.to_c()), 1 if gradient else 0, int(nsrc), int(nrec_sel), int(nfreqs),
                           C.byref(out))
    if rc:
        raise SeisCLEngineError(rc, "footprint: unsupported configuration")
    return int(out.value)


def device_memory():
    """(free, total) bytes of the current CUDA device."""
    lib = load_library()
    f, t = C.c_int64(0), C.c_int64(0)
    rc = lib.sfd_device_memory(C.byref(f), C.byref(t))
    if rc:
        raise SeisCLEngineError(rc, "cudaMemGetInfo failed")
    return int(f.value), int(t.value)


def release_memory():
    """Return the device memory no plan holds (plans allocate from the
    device's pool, which keeps freed memory for the next plan)."""
    rc = load_library().sfd_release_memory()
    if rc:
        raise SeisCLEngineError(rc, "cudaMemPoolTrimTo failed")
