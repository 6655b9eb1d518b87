"""Benchmark of the FDTD forward path on B200.

Workload (default): 3D viscoelastic forward, 8th-order staggered FD, L=2
relaxation mechanisms at constant Q=50 over 5-40 Hz, 256^3 grid, dh=10 m,
dt=1 ms, NT=1500, six flat layers (vp 1800-4200 m/s, vs=vp/1.8, Gardner
density), 20-cell CPML, free surface, a vertical-force Ricker source (10 Hz)
at the grid centre top, 64x64 receivers at 4-cell spacing recording vx, vy,
vz.  Synthetic seeded inputs; layer vp is capped at 4200 m/s because 4500 m/s
violates the CFL limit at dh=10 m, dt=1 ms.

One "step" = one shot = NT time steps of the whole grid.  Metric:
Gcell-updates/s = nz*ny*nx*NT*shots / time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs its own shots on its own GPU (shot sharding,
no data-path collective); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # 3D viscoelastic forward (the metric's headline configuration)
    "visco3d": dict(nd=3, nz=256, ny=256, nx=256, nt=1500, dh=10.0, dt=1e-3, L=2, fdorder=8, nab=20,
                    freesurf=1, f0=10.0, q=50.0, fband=(5.0, 40.0), src_type=2, src_f=10.0),
    # 2D P-SV elastic forward (CPU-runnable case)
    "psv2d": dict(nd=2, nz=300, nx=400, ny=1, nt=2000, dh=10.0, dt=1e-3, L=0, fdorder=8, nab=20, freesurf=1,
                  f0=15.0, src_type=100, src_f=15.0),
}


# Gradient workloads (one "step" = one shot: forward with saved boundaries,
# L2 residual against observed data, res_scale, adjoint, gradient accumulation)
GRADIENT_WORKLOADS = {
    # 2D acoustic FWI gradient, run as 2D P-SV with vs = 0 (the reference's acoustic
    # kernels have no adjoint): 300 x 1000, 4th order, 32 shots, 500 receivers
    "fwi2d": dict(nd=2, nz=300, ny=1, nx=1000, nt=3000, dh=10.0, dt=1e-3, L=0, fdorder=4, nab=20, freesurf=0,
                  f0=8.0, src_type=100, src_f=8.0, precision="fp32", nshots=32, outputs=["p"]),
    # 3D elastic FWI gradient: 200 x 400 x 400, 8th order, saved boundaries in BF16
    # (91.8 GB; FP32 would need 183.5 GB), 16 force shots, 100 x 100 receivers
    "fwi3d": dict(nd=3, nz=200, ny=400, nx=400, nt=2500, dh=12.5, dt=1e-3, L=0, fdorder=8, nab=20, freesurf=1,
                  f0=12.0, src_type=2, src_f=12.0, precision="bf16", nshots=16, outputs=["vx", "vy", "vz"]),
}


def build_gradient_workload(name, nshots, grid=0):
    """Seeded true and starting models and ``nshots`` shots (the workload's
    shot positions, repeated when more are asked for); grid > 0 replaces a 3D
    workload's grid with grid^3 cells (profiling runs)."""
    from scipy.ndimage import gaussian_filter

    w = dict(GRADIENT_WORKLOADS[name])
    if grid > 0 and w["nd"] == 3:
        w["nz"] = w["ny"] = w["nx"] = int(grid)
    w["fl"] = [w["f0"]]
    nd, nz, ny, nx, dh = w["nd"], w["nz"], w["ny"], w["nx"], w["dh"]
    z = np.arange(nz, dtype=np.float64)
    if nd == 2:
        vp = np.broadcast_to(1500.0 + 2500.0 * z / (nz - 1), (nx, nz)).copy()
        rng = np.random.default_rng(301)
        xx, zz = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
        for sgn in (1.0, -1.0):
            cx, cz = rng.uniform(0.25 * nx, 0.75 * nx), rng.uniform(0.3 * nz, 0.7 * nz)
            vp *= 1.0 + 0.1 * sgn * np.exp(-((xx - cx) ** 2 + (zz - cz) ** 2) / (2 * 20.0 ** 2))
        vs = np.zeros_like(vp)
        xs = np.linspace(w["nab"] + 5, nx - w["nab"] - 5, w["nshots"])
        gx = np.linspace(w["nab"], nx - w["nab"] - 1, 500).astype(int)
        shots = []
        for i in range(nshots):
            sp = np.array([[xs[i % w["nshots"]] * dh, 0, 5 * dh, i, w["src_type"]]], np.float32)
            rp = np.zeros((len(gx), 8), np.float32)
            rp[:, 0] = gx * dh
            rp[:, 2] = 5 * dh
            rp[:, 3] = i
            rp[:, 4] = np.arange(1, len(gx) + 1)
            shots.append((sp, ricker(w["src_f"], w["nt"], w["dt"])[None, :], rp))
    else:
        depths = np.sort(np.random.default_rng(401).choice(np.arange(10, nz - 10), 5, replace=False))
        vps = np.sort(np.random.default_rng(401).uniform(1800.0, 4500.0, 6))
        vp1 = np.empty(nz)
        edges = [0] + list(depths) + [nz]
        for l in range(6):
            vp1[edges[l]:edges[l + 1]] = vps[l]
        vp = np.broadcast_to(vp1, (nx, ny, nz)).copy()
        rng = np.random.default_rng(402)
        xx, yy, zz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij", sparse=True)
        for k in range(3):
            c = rng.uniform(0.3, 0.7, 3) * np.array([nx, ny, nz])
            vp *= 1.0 + 0.08 * (1 if k % 2 == 0 else -1) * np.exp(
                -((xx - c[0]) ** 2 + (yy - c[1]) ** 2 + (zz - c[2]) ** 2) / (2 * 15.0 ** 2))
        vs = vp / 1.8
        nr = 100 if min(nx, ny) >= 400 else min(100, (min(nx, ny) - 3) // 4 + 1)   # smaller grids: what fits
        g = np.arange(nr) * 4 + (min(nx, ny) - 4 * nr) // 2 + 2
        gxx, gyy = np.meshgrid(g, g, indexing="ij")
        shots = []
        for i in range(nshots):
            k = i % w["nshots"]   # the 4 x 4 shot grid, repeated
            cx, cy = (2 * (k % 4) + 1) / 8.0 * nx, (2 * (k // 4) + 1) / 8.0 * ny
            sp = np.array([[cx * dh, cy * dh, 5 * dh, i, w["src_type"]]], np.float32)
            rp = np.zeros((gxx.size, 8), np.float32)
            rp[:, 0] = gxx.ravel() * dh
            rp[:, 1] = gyy.ravel() * dh
            rp[:, 2] = 5 * dh
            rp[:, 3] = i
            rp[:, 4] = np.arange(1, gxx.size + 1)
            shots.append((sp, ricker(w["src_f"], w["nt"], w["dt"])[None, :], rp))
    rho = 310.0 * vp ** 0.25
    true = {k: np.ascontiguousarray(v, dtype=np.float32) for k, v in (("vp", vp), ("vs", vs), ("rho", rho))}
    sig = 15.0 if nd == 2 else 8.0
    start = {k: np.ascontiguousarray(gaussian_filter(v, sig), dtype=np.float32) for k, v in true.items()}
    if nd == 2:
        start["vs"][:] = 0.0
    return w, true, start, shots


def ricker(f0, nt, dt):
    t = np.linspace(-1.5 / f0, (nt - 1) * dt - 1.5 / f0, num=int(nt))
    return ((1.0 - 2.0 * (np.pi ** 2) * (f0 ** 2) * (t ** 2)) * np.exp(-(np.pi ** 2) * (f0 ** 2) * (t ** 2))).astype(
        np.float32)


def build_workload(name, grid=0):
    """Seeded synthetic model and acquisition of a workload (host layout);
    grid > 0 replaces a 3D workload's grid with grid^3 cells (profiling runs;
    the receiver array then covers what fits)."""
    w = dict(WORKLOADS[name])
    if grid > 0 and w["nd"] == 3:
        w["nz"] = w["ny"] = w["nx"] = int(grid)
    nd, nz, ny, nx = w["nd"], w["nz"], w["ny"], w["nx"]
    dh = w["dh"]
    if nd == 3:
        depths = np.sort(np.random.default_rng(201).choice(np.arange(10, nz - 10), 5, replace=False))
        vps = np.sort(np.random.default_rng(202).uniform(1800.0, 4200.0, 6))
        vp1 = np.empty(nz, np.float32)
        edges = [0] + list(depths) + [nz]
        for l in range(6):
            vp1[edges[l]:edges[l + 1]] = vps[l]
        vp = np.broadcast_to(vp1, (nx, ny, nz)).astype(np.float32)
    else:
        from scipy.ndimage import gaussian_filter

        def pert(seed):
            g = gaussian_filter(np.random.default_rng(seed).standard_normal((nx, nz)), 8)
            return g / np.abs(g).max()

        vp = (3500.0 * (1 + 0.05 * pert(101))).astype(np.float32)
    if nd == 3:
        vs = (vp / 1.8).astype(np.float32)
        rho = (310.0 * vp ** 0.25).astype(np.float32)
    else:
        vs = (2000.0 * (1 + 0.05 * pert(102))).astype(np.float32)
        rho = (2000.0 * (1 + 0.05 * pert(103))).astype(np.float32)
    taup = taus = None
    fl = [w["f0"]]
    if w["L"] > 0:
        # FL and tau of SeisCL's constant-Q least-squares fit (Q_tau.py's QTAU
        # over the band, tau_optimize, Q2tau(q))
        from seiscl_b200.qfit import constant_q_band

        fl, tau = constant_q_band(w["L"], w["q"], *w["fband"])
        taup = np.full(vp.shape, tau, np.float32)
        taus = np.full(vp.shape, tau, np.float32)
    nt, dt = w["nt"], w["dt"]
    if nd == 3:
        src_pos = np.array([[nx // 2 * dh, ny // 2 * dh, 5 * dh, 0, w["src_type"]]], np.float32)
        nr = min(64, (min(nx, ny) - 3) // 4 + 1)
        gx, gy = np.meshgrid(np.arange(nr) * 4 + 2, np.arange(nr) * 4 + 2, indexing="ij")
        rec = np.zeros((nr * nr, 8), np.float32)
        rec[:, 0] = gx.ravel() * dh
        rec[:, 1] = gy.ravel() * dh
        rec[:, 2] = 5 * dh
        outputs = ["vx", "vy", "vz"]
    else:
        src_pos = np.array([[200 * dh, 0, 5 * dh, 0, w["src_type"]]], np.float32)
        rec = np.zeros((200, 8), np.float32)
        rec[:, 0] = np.arange(200) * 2 * dh
        rec[:, 2] = 5 * dh
        outputs = ["vx", "vz"]
    rec[:, 4] = np.arange(1, rec.shape[0] + 1)
    src = ricker(w["src_f"], nt, dt)[None, :]
    w["fl"] = fl
    return w, dict(vp=vp, vs=vs, rho=rho, taup=taup, taus=taus), dict(src_pos=src_pos, src=src, rec_pos=rec,
                                                                        outputs=outputs)


def engine_config(w):
    from seiscl_b200.engine import Config

    N = [w["nz"], w["ny"], w["nx"]] if w["nd"] == 3 else [w["nz"], w["nx"]]
    return Config(N=N, ND=w["nd"], dh=w["dh"], dt=w["dt"], NT=w["nt"], L=w["L"], f0=w["f0"], FL=w["fl"],
                  FDORDER=w["fdorder"], freesurf=w["freesurf"], abs_type=1, nab=w["nab"], VPPML=3500.0,
                  FPML=w["f0"], NPOWER=2.0, K_MAX_CPML=2.0)


def oracle_config(w):
    return dict(nd=w["nd"], nz=w["nz"], ny=w["ny"], nx=w["nx"], nt=w["nt"], dt=w["dt"], dh=w["dh"], nab=w["nab"],
                freesurf=w["freesurf"], L=w["L"], abs_type=1, fdorder=w["fdorder"], f0=w["f0"], fl=w["fl"],
                vppml=3500.0, fpml=w["f0"])


def reference_build_configs():
    """Grids the reference arm runs (prebuilt in place by build())."""
    out = []
    for name in WORKLOADS:
        w, _, _ = build_workload_light(name)
        out.append(oracle_config(w))
    return out


def build_workload_light(name):
    w = dict(WORKLOADS[name])
    if w["L"] > 0:
        from seiscl_b200.qfit import constant_q_band

        w["fl"] = constant_q_band(w["L"], w["q"], *w["fband"])[0]
    else:
        w["fl"] = [w["f0"]]
    return w, None, None


def algorithmic_bytes(w, state_bytes=4, mem_bytes=None):
    """Minimum DRAM bytes of one time step of the two stencil kernels (FP32).

    Velocity kernel: read 6 stresses, read+write 3 velocities, read 3
    buoyancies; stress kernel: read 3 velocities, read+write 6 stresses and
    6L memory variables, read 5 (elastic) or 10 (viscoelastic) parameters;
    plus read+write of each CPML array cell updated in the absorbing slabs.
    The fused single-pass minimum (each field once) is reported beside."""
    nz, ny, nx, L, nab = w["nz"], w["ny"], w["nx"], w["L"], w["nab"]
    n = nz * ny * nx
    nd = w["nd"]
    if nd == 3:
        nv, ns = 3, 6
        npar_s = 5 if L == 0 else 10
        zlayers = nab if w["freesurf"] else 2 * nab
        psi_cells_axis = 2 * nab * ny * nz + nx * 2 * nab * nz + nx * ny * zlayers
        psi_v = 3 * psi_cells_axis  # psi arrays touched by the velocity update
        psi_s = 3 * psi_cells_axis
    else:
        nv, ns = 2, 3
        npar_s = 3 if L == 0 else 6
        zlayers = nab if w["freesurf"] else 2 * nab
        psi_cells_axis = 2 * nab * nz + nx * zlayers
        psi_v = 2 * psi_cells_axis
        psi_s = 2 * psi_cells_axis
    sb = state_bytes  # bytes per stored wave-field value; parameters and psi stay FP32
    mb = sb if mem_bytes is None else mem_bytes   # bytes per stored memory-variable value
    v_bytes = n * (sb * (ns + 2 * nv) + 4 * nv) + 8 * psi_v
    s_bytes = n * (sb * (nv + 2 * ns) + mb * 2 * ns * L + 4 * npar_s) + 8 * psi_s
    fused = n * (sb * 2 * (nv + ns) + mb * 2 * ns * L + 4 * (nv + npar_s)) + 8 * (psi_v + psi_s)
    return dict(v=v_bytes, s=s_bytes, fused=fused, cells=n)


class ClockSampler:
    def __init__(self, path):
        self.path = path
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self, dev_index=0):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines()]
        except Exception:
            return None
        rows = [[c.strip() for c in r] for r in rows if len(r) >= 9 and r[0].strip() == str(dev_index)]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for i, nme in enumerate(names):
                if r[5 + i].lower() == "active":
                    reasons.add(nme)
        loaded = sorted(sm)[len(sm) // 2:] if sm else []
        return {"sm_mhz": float(np.median(loaded)) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def clock_log_path(args, rank):
    """Where the nvidia-smi clock samples of the timed region go: the path
    given by --clock-log (one file per rank), else the system's temporary
    directory."""
    import tempfile

    if args.clock_log:
        root, ext = os.path.splitext(args.clock_log)
        return "%s_r%d%s" % (root, rank, ext or ".csv")
    return os.path.join(tempfile.gettempdir(), "seiscl_b200_clocks_%d_r%d.csv" % (os.getpid(), rank))


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def cpu_baseline(w, model, acq, budget_s=20.0, prefer_ref=True):
    """The reference's kernels on the host cores over a bounded number of
    time steps of the same grid (OpenMP over all threads), from the fastest
    build of them this CPU can run: -O3 -march=native (when the building
    machine's instruction set is available here), else -O3 -march=x86-64-v3,
    else the -O2 pinning build; the C restatement when none was built."""
    from oracle import build as ob
    from oracle.oracle import DEFAULTS, Oracle

    cfg = oracle_config(w)
    full = dict(DEFAULTS)
    full.update(cfg)
    speed, flags = None, None
    if prefer_ref:
        for sp, fl in (("native", "-O3 -march=native -fopenmp"), ("v3", "-O3 -march=x86-64-v3 -fopenmp"),
                       ("pin", "-O2 -ffp-contract=off -fopenmp")):
            path = ob.ref_lib_path(full, sp)
            if os.path.exists(path) and (sp != "native" or ob.native_usable(path)):
                speed, flags = sp, fl
                break
    kind = "reference" if speed else "port"
    o = Oracle(cfg, ref=bool(speed), speed=speed or "pin")
    rc = o.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    if rc:
        raise RuntimeError("oracle rejected the model (%d)" % rc)
    t0 = time.perf_counter()
    o.run_steps(1)
    one = max(time.perf_counter() - t0, 1e-3)
    nsteps = max(1, min(int(budget_s / one), 200))
    t0 = time.perf_counter()
    o.run_steps(nsteps)
    el = time.perf_counter() - t0
    cells = w["nz"] * w["ny"] * w["nx"]
    o.close()
    what = ("the reference's kernel sources built with %s" % flags) if speed else "the C restatement (-O2)"
    return dict(value=cells * nsteps / el / 1e9, unit="Gcell-updates/s", cores=os.cpu_count(), kind=kind,
                sample="%d time steps of the %dx%dx%d grid (velocity, stress and free-surface kernels), %s"
                       % (nsteps, w["nz"], w["ny"], w["nx"], what)), nsteps, el


def run_reference_arm(args, w, model, acq):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    res = []
    info = None
    for i in range(args.warmup + args.steps):
        b, nsteps, el = cpu_baseline(w, model, acq, budget_s=args.ref_budget)
        if i >= args.warmup:
            res.append(b["value"])
        info = b
    val = float(np.mean(res))
    line = {"impl": "reference", "metric": "Gcell-updates/s", "value": val, "unit": "Gcell-updates/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "grid": [w["nz"], w["ny"], w["nx"]], "nt": w["nt"]},
            "cpu_baseline": dict(info, value=val),
            "e2e": {"value": val, "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_gradient(args):
    """Gradient workloads: per step a batch of shots (``--batch``; default 8
    in 2D, 1 in 3D) advanced together: forward (saving boundaries), L2
    residual against observed data, res_scale and adjoint.  Metric counts
    both sweeps: cells * NT * 2 per shot."""
    import dataclasses

    import torch

    from seiscl_b200.engine import Plan

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if world > 1:
        raise SystemExit("gradient workloads run on one GPU per process without torchrun")
    B = args.batch if args.batch > 0 else (8 if GRADIENT_WORKLOADS[args.workload]["nd"] != 3 else 1)
    if args.checkpoint:
        B = 1   # checkpointed gradients run one shot per launch
    elif args.fields == "fp16":
        raise SystemExit("FP16 wave fields in a gradient need --checkpoint K")
    if args.fields == "fp16_mem":
        raise SystemExit("FP16 memory variables cover forward modelling only")
    nuse = (args.warmup + args.steps) * B
    w, true, start, shots = build_gradient_workload(args.workload, nuse, grid=args.grid)
    if args.nt > 0:
        w["nt"] = args.nt
        shots = [(sp, src[:, :args.nt].copy(), rp) for sp, src, rp in shots]
    outs = w["outputs"]
    cfg = dataclasses.replace(engine_config(w), precision=w["precision"], batch=B,
                              checkpoint=args.checkpoint, field_precision=args.fields,
                              kernels=args.kernels if args.kernels in ("fast", "vector") else "fast")
    plan = Plan(cfg)
    plan.set_model(true["vp"], true["vs"], true["rho"])
    obs = []   # observed data, untimed
    for i in range(0, nuse, B):
        obs += plan.forward_batch(shots[i:i + B], outs)
    plan.set_model(start["vp"], start["vs"], start["rho"])
    plan.zero_gradient()

    def one(i):
        group = shots[i * B:(i + 1) * B]
        ds = plan.forward_batch(group, outs, save_boundaries=True)
        ms = plan.last_loop_ms
        adj = [plan.residual_scale(rp, {k: d[k] - obs[i * B + j][k] for k in outs})
               for j, ((sp, src, rp), d) in enumerate(zip(group, ds))]
        plan.adjoint_batch(group, adj)
        return ms + plan.last_loop_ms

    for i in range(args.warmup):
        one(i)
    torch.cuda.synchronize()
    clk = ClockSampler(clock_log_path(args, rank))
    loop_ms = 0.0
    with clk:
        t0 = time.perf_counter()
        for i in range(args.warmup, args.warmup + args.steps):
            loop_ms += one(i)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    g = plan.gradient(transform=True)
    cells = w["nz"] * w["ny"] * w["nx"]
    updates = cells * w["nt"] * 2 * args.steps * B
    rec = shots[0][2].shape[0] * B
    print(json.dumps({
        "metric": "Gcell-updates/s", "value": round(updates / (loop_ms / 1e3) / 1e9, 3), "unit": "Gcell-updates/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(loop_ms / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "grid": [w["nz"], w["ny"], w["nx"]], "nt": w["nt"],
                   "fdorder": w["fdorder"], "boundaries": w["precision"], "field_storage": args.fields,
                   "outputs": outs,
                   "batch": B,
                   "recompute": ("snapshots every %d steps" % args.checkpoint) if args.checkpoint
                   else "saved boundaries, backpropagation",
                   "step": "%d shot(s) advanced together: forward + residual + res_scale + adjoint "
                           "(2 sweeps counted)" % B},
        "e2e": {"value": round(updates / wall / 1e9, 3), "unit": "Gcell-updates/s",
                "h2d_bytes_per_step": int(B * sum(a.nbytes for a in shots[0]) + len(outs) * rec * w["nt"] * 4),
                "d2h_bytes_per_step": int(len(outs) * rec * w["nt"] * 4)},
        "gradient_finite": bool(all(np.isfinite(v).all() for k, v in g.items() if k in ("vp", "rho"))),
        "gpu_launches": None,
        "clocks": clk.summary(0),
    }))


def serving_requests(nreq, seed=501):
    """The service mix (seeded): 70 % forward / 30 % gradient requests; 80 %
    2D grids (nz 100-400, nx 200-1000), 20 % 3D (64-128^3); physics acoustic,
    elastic or viscoelastic (L 1-3); FD order 4 or 8; NT 500-1500; 1-8 Ricker
    shots at 5-20 Hz, 64 receivers; +-10 % random models.  Acoustic gradient
    requests run as P-SV with vs = 0, the reference's route (the reference's
    acoustic kernels have no adjoint); acoustic requests have no free
    surface, elastic and viscoelastic ones do."""
    from seiscl_b200 import serving
    from seiscl_b200.engine import Config
    from seiscl_b200.qfit import band_frequencies, q_to_tau

    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(nreq):
        three = rng.uniform() < 0.2
        physics = ["acoustic", "elastic", "visco"][int(rng.integers(0, 3))]
        L = int(rng.integers(1, 4)) if physics == "visco" else 0
        order = int(rng.choice([4, 8]))
        nt = int(rng.integers(500, 1500))
        f0 = float(rng.uniform(5, 20))
        kind = "gradient" if rng.uniform() < 0.3 else "forward"
        if three:
            n = int(rng.integers(64, 129)) // 2 * 2
            N, shape = [n, n, n], (n, n, n)
        else:
            nz, nx = int(rng.integers(100, 400)) // 2 * 2, int(rng.integers(200, 1000))
            N, shape = [nz, nx], (nx, nz)
        nd = 3 if three else (22 if physics == "acoustic" and kind == "forward" else 2)
        fl = band_frequencies(L, 0.5 * f0, 2.5 * f0) if L else [f0]
        # acoustic media have no free surface: the reference's free-surface
        # adjoint divides by mu, which is zero there
        cfg = Config(N=N, ND=nd, dh=10.0, dt=8e-4, NT=nt, L=L, f0=f0, FL=fl, FDORDER=order,
                     freesurf=0 if physics == "acoustic" else 1, nab=16)
        vp = np.full(shape, 3000.0, np.float32) * (1 + 0.1 * rng.uniform(-1, 1, shape)).astype(np.float32)
        vs = np.zeros(shape, np.float32) if physics == "acoustic" else (vp / 1.8).astype(np.float32)
        m = {"vp": vp, "vs": None if nd == 22 else vs, "rho": np.full(shape, 2000.0, np.float32)}
        if L:
            tau = q_to_tau(50.0, fl, 0.5 * f0, 2.5 * f0)
            m["taup"] = np.full(shape, tau, np.float32)
            m["taus"] = np.full(shape, tau, np.float32)
        nx_ = shape[0]
        shots = []
        for k in range(int(rng.integers(1, 9))):
            x = float(rng.uniform(20, nx_ - 20)) * 10.0
            y = shape[1] // 2 * 10.0 if three else 0.0
            sp = np.array([[x, y, 50.0, k, 100]], np.float32)
            rp = np.zeros((64, 8), np.float32)
            rp[:, 0] = np.linspace(200.0, (nx_ - 20) * 10.0, 64)
            rp[:, 1] = y
            rp[:, 2] = 50.0
            rp[:, 4] = np.arange(1, 65)
            shots.append((sp, ricker(f0, nt, cfg.dt)[None, :], rp))
        obs = [{"vx": np.zeros((64, nt), np.float32), "vz": np.zeros((64, nt), np.float32)} for _ in shots] \
            if kind == "gradient" else None
        reqs.append(serving.Request(cfg, m, shots, ("vx", "vz"), kind, obs, rid=i))
    return reqs


def _serve_stream(reqs, arrivals, workers, plain):
    """Submit the requests at their arrival times; returns (results, wall s,
    admission stats).  plain: one worker, no batching, time loops launched
    step by step (no CUDA graphs), i.e. the shots one after another with
    plain launches."""
    import dataclasses

    from seiscl_b200 import serving

    if plain:
        reqs = [dataclasses.replace(q, config=dataclasses.replace(q.config, loop_graphs="never")) for q in reqs]
    with serving.Server(workers=1 if plain else workers, max_batch=1 if plain else 8) as srv:
        futs = []
        t0 = time.perf_counter()
        for a, q in zip(arrivals, reqs):
            dt = t0 + a - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            futs.append(srv.submit(q))
        res = [f.result() for f in futs]
        wall = time.perf_counter() - t0
        st = srv.stats()
    return res, wall, st


def run_serving(args):
    """Service mix on one GPU: Poisson arrivals (rate --rate) of the
    requests of ``serving_requests``, served by a pool of workers with
    admission by device memory; then the same stream served plainly (one
    request at a time, shots launched step by step).  Reports shots/s and
    latency percentiles of both."""
    import torch

    from seiscl_b200 import serving

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dist = None
    if world > 1:   # one service per GPU, each taking every world-th request of the stream
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    nreq = max(args.steps, 1)
    reqs_all = serving_requests(nreq)
    arrivals_all = np.cumsum(np.random.default_rng(502).exponential(1.0 / args.rate, nreq))
    reqs, arrivals = reqs_all[rank::world], arrivals_all[rank::world]
    nshots = sum(len(q.shots) for q in reqs_all)
    # warm-up: load the library and the CUDA context outside the timed streams
    _serve_stream(reqs[:1], [0.0], 1, False)
    if dist:
        dist.barrier()
    res, wall, st = _serve_stream(reqs, arrivals, args.workers, False)
    pwall = None
    if not args.no_plain:
        if dist:
            dist.barrier()
        pres, pwall, _ = _serve_stream(reqs, arrivals, 1, True)
    lat = np.array([r.latency for r in res], np.float64)
    plat = np.array([r.latency for r in pres], np.float64) if pwall is not None else np.zeros(0)
    if dist:   # walls: the slowest rank; latencies: all requests
        tt = torch.tensor([wall, pwall or 0.0], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        wall, pwall = float(tt[0]), (float(tt[1]) if pwall is not None else None)
        gl, gp = [None] * world, [None] * world
        dist.all_gather_object(gl, lat.tolist())
        dist.all_gather_object(gp, plat.tolist())
        lat = np.concatenate([np.asarray(x, np.float64) for x in gl])
        plat = np.concatenate([np.asarray(x, np.float64) for x in gp])
        dist.destroy_process_group()
        if rank != 0:
            return
    p = serving.percentiles(lat)
    plain = None
    if pwall is not None:
        pp = serving.percentiles(plat)
        plain = {"shots_per_s": round(nshots / pwall, 3), "wall_s": round(pwall, 2),
                 "latency_s": {k: round(v, 3) for k, v in pp.items()},
                 "what": "same request stream, one request and one shot at a time, step-by-step launches (no CUDA graphs)"}
    reqs = reqs_all
    cells = 0.0
    for q in reqs:
        n = float(np.prod(q.config.N))
        cells += n * q.config.NT * len(q.shots) * (2 if q.kind == "gradient" else 1)
    print(json.dumps({
        "metric": "shots/s", "value": round(nshots / wall, 3), "unit": "shots/s", "n_gpus": world,
        "steps": nreq, "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "serving", "requests": nreq, "shots": nshots, "arrival_rate_per_s": args.rate,
                   "workers": args.workers,
                   "mix": "70 % forward / 30 % gradient; 80 % 2D (100-400 x 200-1000), 20 % 3D (64-128^3); "
                          "acoustic / elastic / visco L 1-3; order 4/8; NT 500-1500; 1-8 shots"},
        "requests_per_s": round(nreq / wall, 3), "latency_s": {k: round(v, 3) for k, v in p.items()},
        "wall_s": round(wall, 2), "gcell_updates_per_s": round(cells / wall / 1e9, 3),
        "admission": {k: int(v) for k, v in st.items()},
        "plain": plain,
        "speedup_vs_plain": round(plain["wall_s"] / wall, 3) if plain else None,
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="visco3d",
                    choices=sorted(WORKLOADS) + sorted(GRADIENT_WORKLOADS) + ["serving"])
    ap.add_argument("--fields", default="fp32", choices=["fp32", "fp16", "fp16_mem"],
                    help="storage of wave fields and memory variables (arithmetic is FP32 either way); "
                         "fp16_mem: memory variables alone in FP16")
    ap.add_argument("--rate", type=float, default=20.0, help="serving: request arrival rate (1/s)")
    ap.add_argument("--workers", type=int, default=8,
                    help="serving: worker threads (8: 18.8 shots/s against 18.0 with 4 on the 60-request mix)")
    ap.add_argument("--no-plain", action="store_true", help="serving: skip the plain one-at-a-time arm")
    ap.add_argument("--batch", type=int, default=0, help="gradient workloads: shots per step (0: 8 in 2D, 1 in 3D)")
    ap.add_argument("--checkpoint", type=int, default=0,
                    help="gradient workloads: snapshot every K steps and recompute (0: saved boundaries)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--ref-budget", type=float, default=15.0)
    ap.add_argument("--kernel-reps", type=int, default=20)
    ap.add_argument("--nt", type=int, default=0, help="override NT (profiling runs only)")
    ap.add_argument("--kernels", default="fast", choices=["fast", "fused", "async", "vector", "stream", "tma", "general"],
                    help="3D kernel family (default: the fastest measured)")
    ap.add_argument("--grid", type=int, default=0, help="3D workloads: override the grid with n^3 (profiling "
                    "runs only)")
    ap.add_argument("--clock-log", default="", help="file for the clock samples of the timed region "
                    "(default: the system temporary directory)")
    args = ap.parse_args()
    if args.workload in GRADIENT_WORKLOADS:
        return run_gradient(args)
    if args.workload == "serving":
        return run_serving(args)

    w, model, acq = build_workload(args.workload, grid=args.grid)
    if args.nt > 0:
        w["nt"] = args.nt
        acq["src"] = acq["src"][:, :args.nt].copy()
    if args.impl == "reference":
        return run_reference_arm(args, w, model, acq)

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from seiscl_b200.engine import Plan

    import dataclasses

    plan = Plan(dataclasses.replace(engine_config(w), field_precision=args.fields, kernels=args.kernels))
    plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    sp, src, rp, outs = acq["src_pos"], acq["src"], acq["rec_pos"], acq["outputs"]
    for _ in range(args.warmup):
        plan.forward(sp, src, rp, outs)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = ClockSampler(clock_log_path(args, rank))
    loop_ms = 0.0
    with clk:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            plan.forward(sp, src, rp, outs)
            loop_ms += plan.last_loop_ms
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    if dist:
        tt = torch.tensor([loop_ms, wall], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        loop_ms, wall = float(tt[0]), float(tt[1])
    cells = w["nz"] * w["ny"] * w["nx"]
    total_updates = cells * w["nt"] * args.steps * world
    value = total_updates / (loop_ms / 1e3) / 1e9
    e2e = total_updates / wall / 1e9
    # kernel-level roofline: the fused step kernel where the plan runs it
    # (velocity + stress + free surface in one launch per step), else the
    # dominant stress update
    kv, ks, ksurf, kfused = plan.bench_kernels(args.kernel_reps)
    ab = algorithmic_bytes(w, 2 if args.fields == "fp16" else 4, 2 if args.fields != "fp32" else 4)
    peak, peak_kind = measured_peaks()
    s_gbs = ab["s"] / (ks / 1e3) / 1e9
    v_gbs = ab["v"] / (kv / 1e3) / 1e9
    step_ms = loop_ms / args.steps / w["nt"]
    fused_gbs = ab["fused"] / (step_ms / 1e3) / 1e9
    fam = plan.kernel_family
    fused = bool(plan.fused_step and kfused > 0)
    vec_name = ("k_s3d_q4_pf<%d>" if args.kernels == "fast" and w["L"] > 0 else "k_s3d_q4<%d>") % w["L"]
    kname = {"vector": vec_name, "tma": "k_tma<1,%d,*>" % w["L"],
             "stream": "k_s3d_stream<4,%d%s>" % (w["L"], ",half" if args.fields == "fp16" else ""),
             "register": "k_s3d_fast", "general": "k_s3d", "2d": "k_s2d"}[fam]
    skern = "stress update, %s%s (%s)" % ({"vector": "4-cell vectorised", "tma": "TMA-pipelined",
                                           "stream": "streaming", "register": "register-blocked",
                                           "general": "general", "2d": "general 2D"}[fam],
                                          {"fp16": ", FP16 storage", "fp16_mem": ", FP16 memory variables"}.get(
                                              args.fields, ""), kname)
    if fused:
        kname = "k_fused3d_q4<%d>" % w["L"]
        skern = "fused 3D step: velocity, stress, memory variables, free surface (%s)" % kname
        k_bytes, k_ms = ab["fused"], kfused
    else:
        k_bytes, k_ms = ab["s"], ks
    k_gbs = k_bytes / (k_ms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_%s.json" % args.workload)
    if os.path.exists(tpath):
        # DRAM bytes per launch of the kernel that ran, from an ncu capture
        key = kname if args.fields == "fp32" else kname + "," + args.fields
        traffic = json.load(open(tpath)).get("stress_kernel_bytes_per_launch", {}).get(key)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu, _, _ = cpu_baseline(w, model, acq, budget_s=args.cpu_budget)
        except Exception as e:  # the baseline must not sink the GPU number
            cpu = {"error": str(e)[:200]}
    h2d = sp.nbytes + src.nbytes + rp.nbytes
    d2h = len(outs) * rp.shape[0] * w["nt"] * 4
    checks = (w["nt"] + 63) // 64   # finite checks of the instability detection
    if w["nd"] == 3 and fused:      # sources, fused step, receivers
        launches_per_shot = 3 * w["nt"] + checks
    elif w["nd"] == 3:   # sources, velocity, stress (FP32 4-cell: with the free surface), [surface], receivers
        sep_surface = w["freesurf"] and (fam != "vector" or args.fields == "fp16")
        launches_per_shot = w["nt"] * (4 + (1 if sep_surface else 0)) + checks
    else:   # 2D modelling: update_v and the fused stress/surface/receiver/source launch
        launches_per_shot = 2 * w["nt"] + 1 + checks
    field_gb = cells * 4 * (9 + 6 * w["L"]) / 1e9 if w["nd"] == 3 else cells * 4 * (5 + 3 * w["L"]) / 1e9
    l2 = ("inputs larger than L2 (%.2f GB of fields)" % field_gb if field_gb > 0.126 else
          "working set L2-resident by design (%.1f MB of fields, reread every time step); no flush" % (field_gb * 1e3))
    line = {
        "metric": "Gcell-updates/s",
        "value": round(value, 3),
        "unit": "Gcell-updates/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(loop_ms / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": args.workload, "field_storage": args.fields, "grid": [w["nz"], w["ny"], w["nx"]], "nt": w["nt"], "L": w["L"],
                   "fdorder": w["fdorder"], "nab": w["nab"], "freesurf": w["freesurf"], "shots_per_gpu": args.steps,
                   "l2": l2},
        "e2e": {"value": round(e2e, 3), "unit": "Gcell-updates/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "hbm", "kernel": skern, "achieved": round(k_gbs, 1),
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(k_gbs / peak, 4),
                     "traffic": traffic, "bytes_per_cell": round(k_bytes / cells, 2),
                     "kernel_ms": round(k_ms, 4),
                     "separate_kernels": {"velocity_ms": round(kv, 4), "stress_ms": round(ks, 4),
                                          "surface_ms": round(ksurf, 4), "velocity_gbs": round(v_gbs, 1),
                                          "stress_gbs": round(s_gbs, 1)},
                     "fused_min_bytes_per_cell": round(ab["fused"] / cells, 2),
                     "step_ms": round(step_ms, 4),
                     "step_effective_gbs_fused_basis": round(fused_gbs, 1),
                     "step_frac_fused_basis": round(fused_gbs / peak, 4)},
        "cpu_baseline": cpu,
        "gpu_launches": launches_per_shot * args.steps,
        "clocks": clk.summary(local),
    }
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
