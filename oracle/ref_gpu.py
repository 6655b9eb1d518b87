"""The reference's 3D forward CUDA kernels on the GPU.

TEST INFRASTRUCTURE ONLY: the reference's own GPU code (update_v3D.cl,
update_s3D.cl and surface3D.cl compiled in place for sm_100a by
oracle/build.py:build_ref_gpu), driven on device copies of the arrays an
Oracle holds -- the reference's preprocessing of the model (parameters, CPML
profiles, taper, eta) and the current wave fields, memory variables and CPML
memory.  Device memory comes from torch; the kernels run on torch's current
stream with the reference's launch geometry: 32 x 4 x 4 work-items with a
haloed tile of (32+8) x (4+8) x (4+8) floats in shared memory for the update
kernels (src/Init_OpenCL.c:489-500, src/clprogram.c:760-773), 256 x 1 over
(ny, nx) for the surface kernel (src/clprogram.c:1030-1042, BLOCK_SIZE of
src/F.h:74).  One time step is update_v, update_s, freesurface (pdir 1), the
order of src/time_stepping.c:426-479 without sources.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import build as _build
from .oracle import MEM_IDS, PARAM_IDS, PSI_IDS, WAVE_IDS, holberg

CPML = ["K", "a", "b", "K_half", "a_half", "b_half"]
V_PSI = ["psi_sxx_x", "psi_sxy_x", "psi_sxy_y", "psi_sxz_x", "psi_sxz_z", "psi_syy_y", "psi_syz_y", "psi_syz_z",
         "psi_szz_z"]
S_PSI = ["psi_vx_x", "psi_vx_y", "psi_vx_z", "psi_vy_x", "psi_vy_y", "psi_vy_z", "psi_vz_x", "psi_vz_y", "psi_vz_z"]


# the parity grid of tests/test_reference_gpu_kernels.py (sizes multiples of
# the reference's 32 x 4 x 4 launch; 8-cell CPML, free surface, L = 2)
SMALL = dict(nd=3, nz=64, ny=32, nx=36, nt=10, dt=1e-3, dh=10.0, nab=8, freesurf=1, L=2, abs_type=1, fdorder=8)


def timing_case() -> dict:
    """The benchmarked 3D grid (bench.py's visco3d workload) with 10 steps."""
    import bench

    w, _, _ = bench.build_workload_light("visco3d")
    return dict(bench.oracle_config(w), nt=10)


def full_cfg(cfg: dict) -> dict:
    """cfg with the oracle's defaults filled in, as Oracle(cfg).cfg holds it."""
    from .oracle import DEFAULTS

    out = dict(DEFAULTS)
    out.update(cfg)
    return out


def prebuild() -> list:
    """Build the libraries of the parity grid and the timing grid (needs the
    reference tree; the built files travel with the repository)."""
    out = []
    for cfg in (SMALL, timing_case()):
        c = full_cfg(cfg)
        out.append(_build.build_ref_gpu(c, holberg(c["fdorder"], c["maxrelerror"])))
    return out


class RefGpu:
    def __init__(self, oracle):
        """Device copies of `oracle`'s arrays, for the reference's kernels
        compiled for oracle.cfg's grid."""
        import torch

        c = dict(oracle.cfg)
        F = c["fdorder"] // 2
        if c["nz"] % 32 or c["ny"] % 4 or c["nx"] % 4:
            raise ValueError("the reference's launch needs nz % 32 == 0 and ny, nx multiples of 4")
        self.cfg = c
        self.torch = torch
        self.lib = C.CDLL(_build.build_ref_gpu(c, holberg(c["fdorder"], c["maxrelerror"])))
        for e in ("update_v", "update_s", "freesurface"):
            fn = getattr(self.lib, "ref_gpu_launch_" + e)
            fn.restype = C.c_int
            fn.argtypes = [C.POINTER(C.c_uint), C.POINTER(C.c_uint), C.c_uint, C.POINTER(C.c_void_p), C.c_void_p]
        dev = torch.device("cuda")
        dummy = torch.zeros(4, dtype=torch.float32, device=dev)

        def put(a):
            if a is None or np.size(a) == 0:
                return dummy
            return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)

        self.dims = (c["nx"] + 2 * F, c["ny"] + 2 * F, c["nz"] + 2 * F)
        self.w = {n: put(oracle.array("wave", n)) for n in WAVE_IDS}
        L = c.get("L", 0)
        self.r = {n: put(oracle.array("mem", n) if L else None) for n in MEM_IDS}
        self.p = {n: put(oracle.array("param", n)) for n in PARAM_IDS}
        absorb = c.get("abs_type", 1) == 1
        self.psi = {n: put(oracle.array("psi", n) if absorb else None) for n in PSI_IDS}
        self.cp = {(ax, n): put(oracle.array("cpml_" + ax, n) if absorb else None) for ax in "xyz" for n in CPML}
        self.taper = put(oracle.array("taper", "") if c.get("abs_type", 1) == 2 else None)
        self.eta = put(oracle.array("eta", "") if L else None)
        self._keep = []

    # ------------------------------------------------------------ launches
    def _args(self, items):
        objs = []
        for it in items:
            if isinstance(it, int):
                objs.append(C.c_int(it))
            elif it is None:
                objs.append(C.c_void_p(0))
            else:
                objs.append(C.c_void_p(it.data_ptr()))
        arr = (C.c_void_p * len(objs))(*[C.cast(C.pointer(o), C.c_void_p) for o in objs])
        self._keep = [objs, arr]
        return arr

    def _launch(self, entry, grid, block, smem, items):
        g = (C.c_uint * 3)(*grid)
        b = (C.c_uint * 3)(*block)
        stream = self.torch.cuda.current_stream().cuda_stream
        rc = getattr(self.lib, "ref_gpu_launch_" + entry)(g, b, smem, self._args(items), C.c_void_p(stream))
        if rc != 0:
            raise RuntimeError("launch of the reference's %s failed: cudaError %d" % (entry, rc))

    def _coefs(self):
        return [self.cp[(ax, n)] for ax in "xyz" for n in CPML]

    def _update_geometry(self):
        c = self.cfg
        bx, by, bz = _build.GPU_BLOCK
        F = c["fdorder"] // 2
        smem = 4 * (bx + 2 * F) * (by + 2 * F) * (bz + 2 * F)
        return (c["nz"] // bx, c["ny"] // by, c["nx"] // bz), (bx, by, bz), smem

    def update_v(self):
        w, p = self.w, self.p
        grid, block, smem = self._update_geometry()
        self._launch("update_v", grid, block, smem,
                     [0, w["vx"], w["vy"], w["vz"], w["sxx"], w["syy"], w["szz"], w["sxy"], w["syz"], w["sxz"],
                      p["rip"], p["rjp"], p["rkp"], self.taper, *self._coefs(),
                      *[self.psi[n] for n in V_PSI], None])

    def update_s(self):
        w, p, r = self.w, self.p, self.r
        grid, block, smem = self._update_geometry()
        self._launch("update_s", grid, block, smem,
                     [0, 0, w["vx"], w["vy"], w["vz"], w["sxx"], w["syy"], w["szz"], w["sxy"], w["syz"], w["sxz"],
                      p["M"], p["mu"], p["muipjp"], p["mujpkp"], p["muipkp"],
                      r["rxx"], r["ryy"], r["rzz"], r["rxy"], r["ryz"], r["rxz"],
                      p["taus"], p["tausipjp"], p["tausjpkp"], p["tausipkp"], p["taup"], self.eta, None, None,
                      self.taper, *self._coefs(), *[self.psi[n] for n in S_PSI], None])

    def freesurface(self, pdir: int = 1):
        c, w, p, r = self.cfg, self.w, self.p, self.r
        self._launch("freesurface", ((c["ny"] + 255) // 256, c["nx"], 1), (256, 1, 1), 0,
                     [w["vx"], w["vy"], w["vz"], w["sxx"], w["syy"], w["szz"], w["sxy"], w["syz"], w["sxz"],
                      p["M"], p["mu"], r["rxx"], r["ryy"], r["rzz"], p["taus"], p["taup"], self.eta,
                      self.cp[("x", "K")], self.psi["psi_vx_x"], self.cp[("y", "K")], self.psi["psi_vy_y"],
                      self.taper, int(pdir)])

    def step(self, n: int = 1):
        for _ in range(n):
            self.update_v()
            self.update_s()
            if self.cfg.get("freesurf", 0):
                self.freesurface(1)
        self.torch.cuda.synchronize()

    def time_kernels(self, nrep: int = 20):
        """Mean ms per launch of (update_v, update_s, freesurface) with CUDA
        events on the current stream, after two untimed launches of each."""
        t = self.torch
        out = []
        for fn in (self.update_v, self.update_s, lambda: self.freesurface(1)):
            for _ in range(2):
                fn()
            e0, e1 = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(nrep):
                fn()
            e1.record()
            e1.synchronize()
            out.append(e0.elapsed_time(e1) / nrep)
        return out

    def fields(self) -> dict:
        out = {n: a.cpu().numpy() for n, a in self.w.items()}
        if self.cfg.get("L", 0):
            out.update({n: a.cpu().numpy() for n, a in self.r.items()})
        return out
