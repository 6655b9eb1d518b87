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


def ricker(f0, nt, dt):
    t = np.linspace(-1.5 / f0, (nt - 1) * dt - 1.5 / f0, num=int(nt))
    return ((1.0 - 2.0 * (np.pi ** 2) * (f0 ** 2) * (t ** 2)) * np.exp(-(np.pi ** 2) * (f0 ** 2) * (t ** 2))).astype(
        np.float32)


def build_workload(name):
    """Seeded synthetic model and acquisition of a workload (host layout)."""
    w = dict(WORKLOADS[name])
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
        from seiscl_b200.qfit import band_frequencies, q_to_tau

        fl = band_frequencies(w["L"], *w["fband"])
        tau = q_to_tau(w["q"], fl, *w["fband"])
        taup = np.full(vp.shape, tau, np.float32)
        taus = np.full(vp.shape, tau, np.float32)
    nt, dt = w["nt"], w["dt"]
    if nd == 3:
        src_pos = np.array([[nx // 2 * dh, ny // 2 * dh, 5 * dh, 0, w["src_type"]]], np.float32)
        gx, gy = np.meshgrid(np.arange(64) * 4 + 2, np.arange(64) * 4 + 2, indexing="ij")
        rec = np.zeros((64 * 64, 8), np.float32)
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
        from seiscl_b200.qfit import band_frequencies

        w["fl"] = band_frequencies(w["L"], *w["fband"])
    else:
        w["fl"] = [w["f0"]]
    return w, None, None


def algorithmic_bytes(w):
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
    v_bytes = n * 4 * (ns + 2 * nv + nv) + 8 * psi_v
    s_bytes = n * 4 * (nv + 2 * ns + 2 * ns * L + npar_s) + 8 * psi_s
    fused = n * 4 * (2 * (nv + ns + ns * L) + nv + npar_s) + 8 * (psi_v + psi_s)
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


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def cpu_baseline(w, model, acq, budget_s=20.0, prefer_ref=True):
    """The CPU oracle on the host cores over a bounded number of time steps
    of the same grid (OpenMP over all threads)."""
    from oracle import build as ob
    from oracle.oracle import Oracle

    from oracle.oracle import DEFAULTS

    cfg = oracle_config(w)
    full = dict(DEFAULTS)
    full.update(cfg)
    ref = bool(prefer_ref and os.path.exists(ob.ref_lib_path(full)))
    kind = "reference" if ref else "port"
    o = Oracle(cfg, ref=ref)
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
    return dict(value=cells * nsteps / el / 1e9, unit="Gcell-updates/s", cores=os.cpu_count(), kind=kind,
                sample="%d time steps of the %dx%dx%d grid (velocity, stress and free-surface kernels)"
                       % (nsteps, w["nz"], w["ny"], w["nx"])), nsteps, el


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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="visco3d", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--ref-budget", type=float, default=15.0)
    ap.add_argument("--kernel-reps", type=int, default=20)
    ap.add_argument("--nt", type=int, default=0, help="override NT (profiling runs only)")
    args = ap.parse_args()

    w, model, acq = build_workload(args.workload)
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

    plan = Plan(engine_config(w))
    plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    sp, src, rp, outs = acq["src_pos"], acq["src"], acq["rec_pos"], acq["outputs"]
    for _ in range(args.warmup):
        plan.forward(sp, src, rp, outs)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = ClockSampler(os.path.join(ROOT, "gpurun_out" if os.path.isdir(os.path.join(ROOT, "gpurun_out"))
                                    else "/tmp", "clocks_bench_r%d.csv" % rank))
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
    # kernel-level roofline (dominant kernel = stress update)
    kv, ks, ksurf = plan.bench_kernels(args.kernel_reps)
    ab = algorithmic_bytes(w)
    peak, peak_kind = measured_peaks()
    s_gbs = ab["s"] / (ks / 1e3) / 1e9
    v_gbs = ab["v"] / (kv / 1e3) / 1e9
    step_ms = loop_ms / args.steps / w["nt"]
    fused_gbs = ab["fused"] / (step_ms / 1e3) / 1e9
    skern = ("stress update, TMA-pipelined (k_tma<1,%d,*>)" % w["L"]) if plan.uses_tma else \
        ("stress update, general (k_s%dd)" % (3 if w["nd"] == 3 else 2))
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_%s.json" % args.workload)
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get("stress_kernel_bytes_per_launch")
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu, _, _ = cpu_baseline(w, model, acq, budget_s=args.cpu_budget)
        except Exception as e:  # the baseline must not sink the GPU number
            cpu = {"error": str(e)[:200]}
    h2d = sp.nbytes + src.nbytes + rp.nbytes
    d2h = len(outs) * rp.shape[0] * w["nt"] * 4
    launches_per_shot = w["nt"] * (4 + (1 if w["freesurf"] else 0))
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
        "config": {"workload": args.workload, "grid": [w["nz"], w["ny"], w["nx"]], "nt": w["nt"], "L": w["L"],
                   "fdorder": w["fdorder"], "nab": w["nab"], "freesurf": w["freesurf"], "shots_per_gpu": args.steps,
                   "l2": "inputs larger than L2 (%.2f GB of fields)" % (cells * 4 * (9 + 6 * w["L"]) / 1e9)},
        "e2e": {"value": round(e2e, 3), "unit": "Gcell-updates/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "hbm", "kernel": skern, "achieved": round(s_gbs, 1),
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(s_gbs / peak, 4),
                     "traffic": traffic, "bytes_per_cell": round(ab["s"] / cells, 2),
                     "velocity_kernel_gbs": round(v_gbs, 1), "kernel_ms": [round(kv, 4), round(ks, 4),
                                                                           round(ksurf, 4)],
                     "fused_min_bytes_per_cell": round(ab["fused"] / cells, 2),
                     "step_effective_gbs_fused_basis": round(fused_gbs, 1)},
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
