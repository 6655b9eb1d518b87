"""Small seeded cases shared by the parity tests (sizes the CPU oracle runs
in seconds).  Models follow SeisCL's host layout: [nx][nz] or [nx][ny][nz]."""
from __future__ import annotations

import numpy as np


def ricker(f0, nt, dt):
    # SeisCL.ricker_wavelet (SeisCL.py:810-834) with tmin = -1.5/f0
    t = np.linspace(-1.5 / f0, (nt - 1) * dt - 1.5 / f0, num=int(nt))
    return ((1.0 - 2.0 * (np.pi ** 2) * (f0 ** 2) * (t ** 2)) * np.exp(-(np.pi ** 2) * (f0 ** 2) * (t ** 2))).astype(
        np.float32)


def make_case(nd=2, nz=48, nx=56, ny=40, nt=200, nab=10, freesurf=1, L=0, abs_type=1, fdorder=8, seed=0,
              src_type=100, dh=10.0, dt=1e-3, f0=15.0, nrec=None):
    rng = np.random.default_rng(seed)
    shape = (nx, ny, nz) if nd == 3 else (nx, nz)
    vp = (3000.0 * (1 + 0.05 * rng.uniform(-1, 1, shape))).astype(np.float32)
    vs = (vp / 1.8).astype(np.float32)
    rho = (2000.0 * (1 + 0.05 * rng.uniform(-1, 1, shape))).astype(np.float32)
    taup = (0.04 + 0.01 * rng.uniform(0, 1, shape)).astype(np.float32) if L else None
    taus = (0.05 + 0.01 * rng.uniform(0, 1, shape)).astype(np.float32) if L else None
    cfg = dict(nd=nd, nz=nz, nx=nx, ny=ny if nd == 3 else 1, nt=nt, dt=dt, dh=dh, nab=nab, freesurf=freesurf,
               L=L, abs_type=abs_type, fdorder=fdorder, f0=f0, fl=[8.0, 30.0, 60.0][:max(L, 1)])
    zs = (nab + 6) * dh if not freesurf else 6 * dh
    ysrc = (ny // 2) * dh if nd == 3 else 0.0
    src_pos = np.array([[(nx // 2) * dh, ysrc, zs, 0, src_type]], np.float32)
    src = ricker(f0, nt, dt)[None, :]
    xs = np.arange(nab + 2, nx - nab - 2, 3)
    if nrec:
        xs = xs[:nrec]
    rec_pos = np.zeros((len(xs), 8), np.float32)
    rec_pos[:, 0] = xs * dh
    rec_pos[:, 1] = ysrc
    rec_pos[:, 2] = zs + 4 * dh
    rec_pos[:, 3] = 0
    rec_pos[:, 4] = np.arange(1, len(xs) + 1)
    return cfg, dict(vp=vp, vs=vs, rho=rho, taup=taup, taus=taus), dict(src_pos=src_pos, src=src, rec_pos=rec_pos)


def engine_config(cfg):
    from seiscl_b200.engine import Config

    N = [cfg["nz"], cfg["ny"], cfg["nx"]] if cfg["nd"] == 3 else [cfg["nz"], cfg["nx"]]
    return Config(N=N, ND=cfg["nd"], dh=cfg["dh"], dt=cfg["dt"], NT=cfg["nt"], L=cfg["L"], f0=cfg["f0"],
                  FL=cfg["fl"], FDORDER=cfg["fdorder"], freesurf=cfg["freesurf"], abs_type=cfg["abs_type"],
                  nab=cfg["nab"], VPPML=3500.0, FPML=15.0, NPOWER=2.0, K_MAX_CPML=2.0, abpc=6.0)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.sqrt(np.sum(b * b))
    return float(np.sqrt(np.sum((a - b) ** 2)) / (den if den > 0 else 1.0))
