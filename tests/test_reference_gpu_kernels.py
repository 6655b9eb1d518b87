"""The reference's own 3D CUDA kernels on the B200.

oracle/ref_gpu.py drives the reference's update_v3D.cl, update_s3D.cl and
surface3D.cl, compiled in place for sm_100a (oracle/build.py:build_ref_gpu,
prebuilt by __graft_entry__.build() where the reference tree is present), on
device copies of the oracle's arrays, with the reference's launch geometry.

* CPU: the built library exports a launcher per kernel.
* GPU parity: from one random state (wave fields and memory variables; CPML
  memory zero) on a 64 x 32 x 36 viscoelastic grid (L = 2, 8-cell CPML,
  free surface), 6 time steps (update_v, update_s, freesurface) of the
  reference's GPU kernels agree with the oracle's, and with this package's
  default kernels on the same state (relative L2 per field below 1e-5).
* GPU timing at the benchmarked grid (256^3, L = 2, 20-cell CPML, free
  surface): the reference's kernels and this package's default kernels per
  launch, on the same GPU in the same process, appended to
  SEISCL_PARITY_REPORT when it is set; this package's step must be faster.
"""
import dataclasses
import json
import os

import numpy as np
import pytest

from tests._cases import engine_config, make_case, rel_l2

NAMES = ["vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "syz", "sxz"]
MEMS = ["rxx", "ryy", "rzz", "rxy", "ryz", "rxz"]
STEPS = 6


def _lib_or_skip(cfg):
    from oracle import build
    from oracle.oracle import holberg
    from oracle.ref_gpu import full_cfg

    c = full_cfg(cfg)
    path = build.ref_gpu_lib_path(c)
    if not os.path.exists(path):
        if not build.ref_available():
            pytest.skip("the reference's GPU kernels were not prebuilt and the reference tree is absent")
        build.build_ref_gpu(c, holberg(c["fdorder"], c["maxrelerror"]))
    return path


def test_reference_gpu_library_exports_launchers():
    import ctypes

    from oracle.ref_gpu import SMALL

    lib = ctypes.CDLL(_lib_or_skip(SMALL))
    for e in ("update_v", "update_s", "freesurface"):
        assert getattr(lib, "ref_gpu_launch_" + e) is not None


def _report(**kw):
    path = os.environ.get("SEISCL_PARITY_REPORT")
    if path:
        with open(path, "a") as fh:
            fh.write(json.dumps(kw) + "\n")


def _state(cfg, par_scale, seed):
    """Random interior wave fields (velocities ~ sqrt(buoyancy), stresses ~
    sqrt(M)) and memory variables, in the padded layout."""
    rng = np.random.default_rng(seed)
    F = cfg["fdorder"] // 2
    dims = (cfg["nx"] + 2 * F, cfg["ny"] + 2 * F, cfg["nz"] + 2 * F)
    sl = tuple(slice(F, d - F) for d in dims)
    out = {}
    for n in NAMES:
        a = np.zeros(dims, np.float32)
        s = par_scale["v"] if n[0] == "v" else par_scale["s"]
        a[sl] = rng.uniform(-1.0, 1.0, a[sl].shape) * s
        out[n] = a.ravel()
    for n in MEMS:
        a = np.zeros((cfg["L"],) + dims, np.float32)
        a[(slice(None),) + sl] = rng.uniform(-1.0, 1.0, a[(slice(None),) + sl].shape) * par_scale["s"] * 1e-3
        out[n] = a.ravel()
    return out


@pytest.mark.gpu
def test_reference_gpu_kernels_match_oracle_and_this_package(cuda_device):
    from oracle.oracle import Oracle
    from oracle.ref_gpu import SMALL, RefGpu
    from seiscl_b200.engine import Plan

    _lib_or_skip(SMALL)
    kw = {k: SMALL[k] for k in ("nd", "nz", "ny", "nx", "nt", "nab", "freesurf", "L", "abs_type", "fdorder")}
    cfg, model, acq = make_case(seed=31, **kw)
    ora = Oracle(cfg)
    assert ora.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"]) == 0
    par = {"v": float(np.sqrt(ora.array("param", "rip").mean())), "s": float(np.sqrt(ora.array("param", "M").mean()))}
    init = _state(cfg, par, 5)
    for n in NAMES:
        ora.set_array("wave", n, init[n])
    for n in MEMS:
        ora.set_array("mem", n, init[n])
    ref = RefGpu(ora)
    ref.step(STEPS)
    got_ref = ref.fields()
    ora.run_steps(STEPS)

    plan = Plan(engine_config(cfg))
    plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    # a source-free forward leaves every field and CPML memory at zero
    plan.forward(acq["src_pos"], acq["src"] * 0, acq["rec_pos"], ["vx"])
    for i, n in enumerate(NAMES):
        plan.debug_load(0, i, init[n])
    for i, n in enumerate(MEMS):
        plan.debug_load(2, i, init[n])
    for _ in range(STEPS):
        for k in (0, 1, 2):
            plan.debug_launch(k)
    ours = {n: plan.debug_array(0, i, plan.nvol) for i, n in enumerate(NAMES)}
    ours.update({n: plan.debug_array(2, i, plan.nvol * cfg["L"]) for i, n in enumerate(MEMS)})
    plan.close()

    for n in NAMES + MEMS:
        kind = "wave" if n in NAMES else "mem"
        o = ora.array(kind, n)
        assert np.abs(o).max() > 0, n
        e_ora = rel_l2(got_ref[n], o)
        e_ours = rel_l2(ours[n], got_ref[n])
        _report(case="reference GPU kernels 64x32x36 L2 %d steps" % STEPS, field=n, ref_gpu_vs_oracle=e_ora,
                ours_vs_ref_gpu=e_ours)
        assert e_ora < 1e-5, (n, e_ora)
        assert e_ours < 1e-5, (n, e_ours)
    ora.close()


@pytest.mark.gpu
def test_reference_gpu_kernels_timed_beside_this_package(cuda_device):
    import bench
    from oracle.oracle import Oracle
    from oracle.ref_gpu import RefGpu, timing_case
    from seiscl_b200.engine import Plan

    cfg = timing_case()
    _lib_or_skip(cfg)
    w, model, _ = bench.build_workload("visco3d")
    ora = Oracle(cfg)
    assert ora.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"]) == 0
    ref = RefGpu(ora)
    ora.close()
    rv, rs, rf = ref.time_kernels(10)
    del ref
    plan = Plan(dataclasses.replace(bench.engine_config(w), NT=10))
    plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    plan.bench_kernels(3)
    ov, os_, osurf, _ = plan.bench_kernels(10)
    plan.close()
    ref_step = rv + rs + rf
    ours_step = ov + os_   # the free surface runs inside the stress update
    _report(case="reference GPU kernels vs this package, visco3d 256^3 L2 CPML20 free surface",
            ref_update_v_ms=rv, ref_update_s_ms=rs, ref_freesurface_ms=rf, ref_step_ms=ref_step,
            ours_velocity_ms=ov, ours_stress_ms=os_, ours_separate_surface_ms=osurf, ours_step_ms=ours_step,
            speedup=ref_step / ours_step)
    print("REFGPU update_v %.4f update_s %.4f surface %.4f | ours v %.4f s %.4f | step %.4f vs %.4f (%.2fx)"
          % (rv, rs, rf, ov, os_, ref_step, ours_step, ref_step / ours_step))
    assert ours_step < ref_step
