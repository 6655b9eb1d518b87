"""Edge cases of a shot: empty and ragged point lists, points outside the
grid, the shortest runs, and a job larger than the device.

SeisCL maps a source or receiver to the cell (int)(x/dh) + fdoh along each
axis and skips it when that cell lies outside [fdoh, NX - fdoh - 1] along x
(automatic_kernels.c:501-511 for the sources; the receiver kernels test the
same range).  A point inside that x range but outside the padded grid along
y or z indexes memory outside the wave fields in SeisCL; this package refuses
such a shot with SFD_ERR_ARG and leaves the plan usable.

* CPU: the oracle drops the points outside the x range (the seismograms of
  the shot with them equal those of the shot without them, bit for bit, and
  their traces stay zero) and returns empty seismograms for a shot without
  receivers.
* GPU, through the C ABI: the same shots against the oracle (forward
  tolerance of the parity tests); a shot without receivers or without
  sources; a gradient shot without receivers (against the oracle: SeisCL's
  adjoint starts from the forward's CPML memory, so it is not zero); a batch
  mixing such shots with ordinary ones, bit for bit against
  single runs; runs of 1, 2 and 3 time steps; the refusal of points outside
  the padded grid; and a gradient job whose saved boundaries exceed the
  device's memory, refused with SFD_ERR_MEMORY without losing the plan.
"""
import dataclasses

import numpy as np
import pytest

from tests._cases import engine_config, make_case, rel_l2

FWD_TOL = 2e-5   # the forward tolerance of tests/test_gpu_parity.py
GRAD_TOL = 2e-4  # and its raw-gradient tolerance
SFD_ERR_ARG = -1
SFD_ERR_MEMORY = -4

CASE_2D = dict(nd=2, freesurf=1, L=0, abs_type=1, src_type=100, nt=120, seed=71)
CASE_3D = dict(nd=3, freesurf=0, L=1, abs_type=1, src_type=100, nz=36, ny=34, nx=38, nt=80, nab=8, seed=72)


def _outputs(nd):
    return ["vx", "vy", "vz", "p"] if nd == 3 else ["vx", "vz", "p"]


def _with_outside_points(cfg, acq):
    """The case's shot plus sources and receivers outside the x range of the
    interior, and receivers just inside it.  Returns (src_pos, src, rec_pos,
    inside) with ``inside`` the receivers' mask."""
    dh, nx, nz = cfg["dh"], cfg["nx"], cfg["nz"]
    F = cfg["fdorder"] // 2
    sp = acq["src_pos"]
    y = sp[0, 1]
    extra_src = np.array([[(nx + 2) * dh, y, sp[0, 2], 1, sp[0, 4]],    # cell nx + 2 + F: beyond the interior
                          [-2.0 * dh, y, sp[0, 2], 2, sp[0, 4]]], np.float32)   # cell F - 2: in the padding
    src_pos = np.concatenate([sp, extra_src])
    src = np.concatenate([acq["src"], 0.7 * acq["src"], -1.3 * acq["src"]]).astype(np.float32)
    zr = acq["rec_pos"][0, 2]
    # x positions: (int)(x/dh) truncates toward zero, so -0.5 dh maps to the
    # first interior cell and -1 dh to the padding
    xs = [-1.0 * dh, -0.5 * dh, 3.0 * dh, (nx - 1) * dh, nx * dh, (nx + 5) * dh, -7.0 * dh]
    inside = np.array([False, True, True, True, False, False, False])
    rec = np.zeros((len(xs) + 1, 8), np.float32)
    rec[:-1, 0] = xs
    rec[:, 1] = y
    rec[:-1, 2] = zr
    # one receiver in the z padding above the grid (cell F - 2 >= 0): inside
    # the padded fields, so it records what the padding holds
    rec[-1, 0] = (nx // 3) * dh
    rec[-1, 2] = -2.0 * dh
    rec[:, 4] = np.arange(1, len(rec) + 1)
    assert F >= 2 and nz > 4
    return src_pos, src, rec, np.append(inside, True)


def test_oracle_drops_points_outside_the_interior():
    from oracle.oracle import Oracle

    cfg, model, acq = make_case(**dict(CASE_2D, nt=60))
    outs = _outputs(cfg["nd"])
    ora = Oracle(cfg)
    assert ora.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"]) == 0
    src_pos, src, rec, inside = _with_outside_points(cfg, acq)
    d_all = ora.forward(src_pos, src, rec, outs)
    d_in = ora.forward(src_pos[:1], src[:1], rec[inside], outs)
    for n in outs:
        assert np.array_equal(d_all[n][inside], d_in[n]), n
        assert not np.any(d_all[n][~inside]), n
    assert np.abs(d_in["vz"]).max() > 0
    d0 = ora.forward(acq["src_pos"], acq["src"], np.zeros((0, 8), np.float32), outs)
    for n in outs:
        assert d0[n].shape == (0, cfg["nt"]), n
    ora.close()


def _plan(cfg, model, **over):
    from seiscl_b200.engine import Plan

    plan = Plan(dataclasses.replace(engine_config(cfg), **over))
    plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    return plan


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [CASE_2D, CASE_3D], ids=["psv2d", "visco3d"])
def test_points_outside_the_interior_are_dropped(kw, cuda_device):
    from oracle.oracle import Oracle

    cfg, model, acq = make_case(**kw)
    outs = _outputs(cfg["nd"])
    src_pos, src, rec, inside = _with_outside_points(cfg, acq)
    ora = Oracle(cfg)
    assert ora.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"]) == 0
    d_ref = ora.forward(src_pos, src, rec, outs)
    ora.close()
    plan = _plan(cfg, model)
    d_all = plan.forward(src_pos, src, rec, outs)
    d_in = plan.forward(src_pos[:1], src[:1], rec[inside], outs)
    plan.close()
    for n in outs:
        assert np.abs(d_ref[n]).max() > 0, n
        assert rel_l2(d_all[n], d_ref[n]) < FWD_TOL, (n, rel_l2(d_all[n], d_ref[n]))
        assert not np.any(d_all[n][~inside]), n
        # the dropped points change nothing on the device either
        assert np.array_equal(d_all[n][inside], d_in[n]), n


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [CASE_2D, CASE_3D], ids=["psv2d", "visco3d"])
def test_shot_without_receivers_or_sources(kw, cuda_device):
    cfg, model, acq = make_case(**kw)
    outs = _outputs(cfg["nd"])
    nt = cfg["nt"]
    plan = _plan(cfg, model)
    want = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
    assert np.abs(want["vz"]).max() > 0
    # no receivers: empty seismograms
    d = plan.forward(acq["src_pos"], acq["src"], np.zeros((0, 8), np.float32), outs)
    for n in outs:
        assert d[n].shape == (0, nt), n
    # no sources: a wave field that stays at rest
    d = plan.forward(np.zeros((0, 5), np.float32), np.zeros((0, nt), np.float32), acq["rec_pos"], outs)
    for n in outs:
        assert d[n].shape == want[n].shape and not np.any(d[n]), n
    # neither leaves a trace in the plan's state
    again = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
    for n in outs:
        assert np.array_equal(again[n], want[n]), n
    plan.close()


@pytest.mark.gpu
def test_gradient_shot_without_receivers(cuda_device):
    """No residual is injected, but SeisCL's adjoint starts from the CPML
    memory the forward run left behind, which seeds a small adjoint field:
    the gradient is the oracle's (parity tolerance), and exactly zero when the
    adjoint starts from zeroed CPML memory."""
    from oracle.oracle import Oracle

    cfg, model, acq = make_case(**CASE_2D)
    nt = cfg["nt"]
    none = np.zeros((0, 8), np.float32)
    res = {"vx": np.zeros((0, nt), np.float32)}
    ora = Oracle(cfg)
    assert ora.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"]) == 0
    ora.forward(acq["src_pos"], acq["src"], none, ["vx"], save_boundaries=True)
    ora.clear_gradients()
    ora.adjoint(acq["src_pos"], acq["src"], none, res)
    g_ref = ora.gradients()
    ora.close()
    for reset in (False, True):
        plan = _plan(cfg, model, adjoint_reset_psi=reset)
        plan.forward(acq["src_pos"], acq["src"], none, ["vx"], save_boundaries=True)
        plan.zero_gradient()
        plan.adjoint(acq["src_pos"], acq["src"], none, res)
        g = plan.gradient(transform=False)
        plan.close()
        for ours, theirs in (("M", "rawM"), ("mu", "rawmu"), ("rho", "rawrho")):
            if reset:
                assert not np.any(g[ours]), ours
            else:
                assert np.abs(g_ref[theirs]).max() > 0, theirs
                assert rel_l2(g[ours], g_ref[theirs]) < GRAD_TOL, (ours, rel_l2(g[ours], g_ref[theirs]))


@pytest.mark.gpu
def test_batch_with_empty_and_dropped_shots(cuda_device):
    """A batch whose shots have 0, all-outside and ordinary receiver lists,
    and a shot whose only source is outside the interior: each shot's
    seismograms equal its single run, bit for bit."""
    cfg, model, acq = make_case(**dict(CASE_2D, seed=73))
    outs = ["vx", "vz", "p"]
    src_pos, src, rec, inside = _with_outside_points(cfg, acq)
    shots = [
        (acq["src_pos"], acq["src"], np.zeros((0, 8), np.float32)),
        (src_pos, src, rec),
        (src_pos[1:2], src[1:2], acq["rec_pos"]),            # its one source dropped: silent
        (acq["src_pos"], (0.5 * acq["src"]).astype(np.float32), rec[~inside]),   # every receiver dropped
    ]
    one = _plan(cfg, model)
    ref = [one.forward(sp, s, rp, outs) for sp, s, rp in shots]
    one.close()
    many = _plan(cfg, model, batch=4)
    got = many.forward_batch(shots, outs)
    many.close()
    assert np.abs(ref[1]["vz"]).max() > 0
    assert not np.any(ref[2]["vz"]) and not np.any(ref[3]["p"])
    for r, g in zip(ref, got):
        for n in outs:
            assert r[n].shape == g[n].shape, n
            assert np.array_equal(r[n], g[n]), (n, float(np.abs(r[n] - g[n]).max()) if r[n].size else 0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("nt", [1, 2, 3])
@pytest.mark.parametrize("kw", [CASE_2D, CASE_3D], ids=["psv2d", "visco3d"])
def test_shortest_runs_match_oracle(kw, nt, cuda_device):
    """Runs of 1 to 3 time steps, with receivers on and around the source
    cell so that the first samples are not zero."""
    from oracle.oracle import Oracle

    cfg, model, acq = make_case(**dict(kw, nt=nt))
    outs = _outputs(cfg["nd"])
    rng = np.random.default_rng(nt)
    src = rng.standard_normal((1, nt)).astype(np.float32)
    dh = cfg["dh"]
    sx, sy, sz = acq["src_pos"][0, :3]
    rec = np.zeros((5, 8), np.float32)
    rec[:, 0] = sx + dh * np.array([0, 1, -1, 0, 2])
    rec[:, 1] = sy
    rec[:, 2] = sz + dh * np.array([0, 0, 0, 1, 3])
    rec[:, 4] = np.arange(1, 6)
    ora = Oracle(cfg)
    assert ora.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"]) == 0
    d_ref = ora.forward(acq["src_pos"], src, rec, outs)
    ora.close()
    plan = _plan(cfg, model)
    d = plan.forward(acq["src_pos"], src, rec, outs)
    plan.close()
    assert np.abs(d_ref["p"]).max() > 0
    for n in outs:
        assert d[n].shape == (5, nt), n
        assert rel_l2(d[n], d_ref[n]) < FWD_TOL, (n, rel_l2(d[n], d_ref[n]))


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [CASE_2D, CASE_3D], ids=["psv2d", "visco3d"])
def test_points_outside_the_padded_grid_are_refused(kw, cuda_device):
    from seiscl_b200.engine import SeisCLEngineError

    cfg, model, acq = make_case(**kw)
    outs = _outputs(cfg["nd"])
    F = cfg["fdorder"] // 2
    dh = cfg["dh"]
    plan = _plan(cfg, model)
    want = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
    bad_rec = acq["rec_pos"].copy()
    bad_rec[1, 2] = -(F + 3) * dh                  # cell -3 along z
    bad_src = acq["src_pos"].copy()
    bad_src[0, 2] = (cfg["nz"] + F + 2) * dh       # cell NZ + 2 along z
    cases = [(acq["src_pos"], bad_rec), (bad_src, acq["rec_pos"])]
    if cfg["nd"] == 3:
        far_y = acq["rec_pos"].copy()
        far_y[0, 1] = (cfg["ny"] + 2 * F) * dh     # cell NY + F along y
        cases.append((acq["src_pos"], far_y))
    for sp, rp in cases:
        with pytest.raises(SeisCLEngineError) as e:
            plan.forward(sp, acq["src"], rp, outs)
        assert e.value.code == SFD_ERR_ARG
        assert "outside the padded grid" in str(e.value)
    again = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)
    plan.close()
    for n in outs:
        assert np.array_equal(again[n], want[n]), n


@pytest.mark.gpu
def test_gradient_job_larger_than_the_device_is_refused(cuda_device):
    """A 2000 x 2000 P-SV gradient job with enough time steps that one saved
    boundary field exceeds the device's memory: the forward run refuses it
    with SFD_ERR_MEMORY before any time step, the device memory comes back,
    and the plan still models (tmax bounds the steps if the refusal were
    ever missed)."""
    import torch

    from seiscl_b200.engine import SeisCLEngineError, footprint

    cfg, model, acq = make_case(**dict(CASE_2D, nz=2000, nx=2000, nab=20, nt=8))
    ec = dataclasses.replace(engine_config(cfg), tmax=2)
    total = torch.cuda.mem_get_info(cuda_device)[1]
    per_step = (footprint(dataclasses.replace(ec, NT=2000), True, 1, 1)
                - footprint(dataclasses.replace(ec, NT=1000), True, 1, 1)) // 1000
    nwave = 5   # P-SV: vx, vz, sxx, szz, sxz
    nt = int(2 * total // (per_step // nwave)) + 1   # one field's store alone is twice the device
    big = dataclasses.replace(ec, NT=nt)
    assert footprint(big, True, 1, 1) > 2 * total
    from seiscl_b200.engine import Plan

    plan = Plan(big)
    plan.set_model(model["vp"], model["vs"], model["rho"], None, None)
    src = np.zeros((1, nt), np.float32)
    src[0, :8] = np.random.default_rng(8).standard_normal(8)
    # receivers on and beside the source cell: nonzero from the first step
    rec = np.zeros((3, 8), np.float32)
    rec[:, 0] = acq["src_pos"][0, 0] + cfg["dh"] * np.array([0, 1, -1])
    rec[:, 2] = acq["src_pos"][0, 2]
    with pytest.raises(SeisCLEngineError) as e:
        plan.forward(acq["src_pos"], src, rec, ["vz"], save_boundaries=True)
    assert e.value.code == SFD_ERR_MEMORY
    # the plan models on: the first tmax samples of a short plan's run
    d = plan.forward(acq["src_pos"], src, rec, ["vz"])
    plan.close()
    small = _plan(cfg, model, tmax=2)
    want = small.forward(acq["src_pos"], src[:, :8], rec, ["vz"])
    small.close()
    assert np.abs(want["vz"][:, :2]).max() > 0
    assert np.array_equal(d["vz"][:, :2], want["vz"][:, :2])
    assert not np.any(d["vz"][:, 2:])
    torch.cuda.synchronize(cuda_device)
    assert torch.cuda.mem_get_info(cuda_device)[0] > total // 2
