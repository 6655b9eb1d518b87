"""The SeisCL-compatible front end (seiscl_b200.seiscl.SeisCL).

CPU tests cover the host logic restated from SeisCL/SeisCL.py and
src/residuals.c / src/butterworth.c (acquisition helpers, data selection,
output names, residuals and misfit, band-pass filter).  GPU tests run whole
jobs through the front end and compare them with the oracle driven the way
src/time_stepping.c drives the reference: forward per shot, L2 residual,
res_scale, adjoint, transf_grad.
"""
import numpy as np
import pytest

from tests._cases import rel_l2, ricker

FWD_TOL = 2e-5
GRAD_TOL = 2e-4


def _seis(**kw):
    from seiscl_b200.seiscl import SeisCL

    args = dict(ND=2, N=np.array([48, 60]), dh=10.0, dt=1e-3, NT=220, nab=10, freesurf=1, f0=15.0,
                FDORDER=8, abs_type=1, seisout=1, workdir="unused")
    args.update(kw)
    return SeisCL(**args)


def _models(N, seed):
    rng = np.random.default_rng(seed)
    vp = (3000.0 * (1 + 0.05 * rng.uniform(-1, 1, N))).astype(np.float32)
    return {"vp": vp, "vs": (vp / 1.8).astype(np.float32),
            "rho": (2000.0 * (1 + 0.05 * rng.uniform(-1, 1, N))).astype(np.float32)}


# ------------------------------------------------------------------ host logic
def test_constructor_defaults_match_reference():
    s = _seis()
    d = __import__("seiscl_b200.seiscl", fromlist=["SeisCL"]).SeisCL()
    assert (d.ND, d.dh, d.dt, d.NT, d.L, d.FDORDER, d.MAXRELERROR, d.nab, d.abpc) == (2, 10, 0.0008, 875, 0, 8, 1, 16, 6)
    assert (d.VPPML, d.NPOWER, d.FPML, d.K_MAX_CPML, d.seisout, d.param_type) == (3500, 2, 15, 2, 2, 0)
    assert d.file_din == "SeisCL_din.mat" and d.file_gout == "SeisCL_gout.mat"
    assert s.params == ["vp", "vs", "rho"]
    s.L = 1
    s.param_type = 1
    assert s.params == ["M", "mu", "rho", "taup", "taus"]


@pytest.mark.parametrize("nd,seisout,names", [
    (2, 1, ["vx", "vz"]), (3, 1, ["vx", "vy", "vz"]), (21, 1, ["vy"]), (2, 2, ["p"]),
    (2, 3, ["sxx", "szz", "sxz"]), (21, 3, ["sxy", "syz"]),
    (3, 4, ["vx", "vy", "vz", "sxx", "syy", "szz", "sxz", "sxy", "syz"]),
])
def test_to_load_names(nd, seisout, names):
    s = _seis(ND=nd, seisout=seisout)
    assert s.to_load_names == names
    s.to_load_names = ["vx"]
    assert s.to_load_names == ["vx"]


def test_surface_acquisition_and_prepare_data():
    s = _seis(N=np.array([60, 100]), nab=16, freesurf=0)
    s.surface_acquisition_2d(dg=4, ds=20, dsx=2, dsz=3, dgsz=1)
    sp, rp = s.src_pos_all, s.rec_pos_all
    xs = np.arange(18, 100 - 18, 20)
    assert np.allclose(sp[0], xs * 10.0) and np.allclose(sp[2], 19 * 10.0)
    assert np.allclose(sp[3], np.arange(len(xs))) and np.all(sp[4] == 100)
    gx = np.arange(20, 100 - 18, 4) * 10.0
    assert rp.shape[1] == len(xs) * len(gx)
    assert np.allclose(rp[0, :len(gx)], gx) and np.allclose(rp[2], 20 * 10.0)
    assert np.allclose(rp[4], np.arange(1, rp.shape[1] + 1))
    s.prepare_data([1, 2])
    assert s.src_pos.shape[1] == 2 and s.rec_pos.shape[1] == 2 * len(gx)
    assert np.allclose(s.rec_pos[4], np.arange(len(gx) + 1, 3 * len(gx) + 1))
    assert s.src.shape == (s.NT, 2)
    # offset filter keeps receivers within [offmin, offmax] of their shot
    s.filter_offset = True
    s.offmax = 100.0
    s.prepare_data(1)
    off = np.abs(s.rec_pos[0] - s.src_pos[0, 0])
    assert len(off) > 0 and np.all(off <= 100.0)
    with pytest.raises(ValueError):
        s.prepare_data(99)


def test_crosshole_acquisition():
    s = _seis(N=np.array([80, 60]), nab=10, freesurf=1)
    s.crosshole_acquisition_2d(dg=3, ds=10, dsx=2, dsz=4)
    sp, rp = s.src_pos_all, s.rec_pos_all
    zs = np.arange(4, 80 - 4, 10)
    assert np.allclose(sp[2], zs * 10.0) and np.allclose(sp[0], 12 * 10.0)
    assert np.allclose(rp[0], (60 - 12) * 10.0) and np.all(rp[5] == 2)
    assert rp.shape[1] == len(zs) * len(np.arange(4, 76, 3))


def test_missing_parameter_and_unread_outputs_raise():
    from seiscl_b200.seiscl import SeisCLError

    s = _seis()
    s.src_pos_all = np.array([[200.0], [0], [60.0], [0], [100]])
    s.rec_pos_all = np.array([[300.0], [0], [60.0], [0], [1], [0], [0], [0]])
    with pytest.raises(SeisCLError):
        s.set_forward(0, {"vp": np.ones((48, 60))})
    with pytest.raises(SeisCLError):
        s.read_data()
    with pytest.raises(SeisCLError):
        s.read_grad()
    with pytest.raises(SeisCLError):
        s.read_rms()


def test_next_fast_size():
    from seiscl_b200.seiscl import next_fast_size

    assert [next_fast_size(n) for n in (1, 7, 11, 13, 17, 875, 1001)] == [1, 8, 12, 15, 18, 900, 1024]


def test_butterworth_matches_loop_restatement():
    """Against a direct transcription of butterworth.c's steps on one trace."""
    from seiscl_b200.seiscl import butterworth, next_fast_size

    rng = np.random.default_rng(3)
    NT, tmax, dt = 300, 250, 1e-3
    d = rng.standard_normal((3, NT)).astype(np.float32)
    got = butterworth(d, 10.0, 60.0, dt, tmax)
    nfft = next_fast_size(tmax)
    for n in range(3):
        buf = np.concatenate([d[n, :tmax], d[n, :nfft - tmax]]).astype(np.float64)
        spec = np.fft.rfft(buf)
        for t in range(nfft // 2 + 1):
            f = t / (dt * nfft)
            H = (1.0 - np.sqrt(1.0 / (1.0 + (f / 10.0) ** 12))) * np.sqrt(1.0 / (1.0 + (f / 60.0) ** 12))
            spec[t] *= H
        want = np.fft.irfft(spec, n=nfft)[:tmax]
        assert np.allclose(got[n, :tmax], want, rtol=1e-5, atol=1e-6)
        assert np.array_equal(got[n, tmax:], d[n, tmax:])
    # a tone inside the band passes, one far outside is removed
    t = np.arange(NT) * dt
    tone = np.stack([np.sin(2 * np.pi * 30.0 * t), np.sin(2 * np.pi * 200.0 * t)]).astype(np.float32)
    out = butterworth(tone, 10.0, 60.0, dt, NT)
    assert np.std(out[0, 50:-50]) > 0.5 * np.std(tone[0])
    assert np.std(out[1, 50:-50]) < 0.01


def _residuals_loops(out, obs, tmin, tmax, scalerms, scalermsnorm, scaleshot):
    """Line-by-line restatement of var_res_raw (residuals.c:58-450) for one
    shot and back_prop_type 1, in float64 loops."""
    names = list(out)
    out = {k: v.astype(np.float64).copy() for k, v in out.items()}
    obs = {k: v.astype(np.float64).copy() for k, v in obs.items()}
    nrec = out[names[0]].shape[0]
    rs, rs0 = np.ones(nrec), np.ones(nrec)
    ws = 0.0
    if scalerms or scaleshot or scalermsnorm:
        for g in range(nrec):
            a = b = 0.0
            for k in names:
                for t in range(tmin, tmax):
                    a += out[k][g, t] ** 2
                    b += obs[k][g, t] ** 2
            rs[g], rs0[g] = np.sqrt(1.0 / a), np.sqrt(1.0 / b)
    if scaleshot:
        ws = 1 / np.sqrt(sum(1 / rs0[g] ** 2 for g in range(nrec)))
        rs[:] = ws
        rs0[:] = ws
    if scalerms:
        ws = 1 / np.sqrt(sum(1 / rs0[g] ** 2 for g in range(nrec)))
        for g in range(nrec):
            rs[g] *= ws / rs0[g]
            rs0[g] = ws
    if scalerms or scaleshot or scalermsnorm:
        for g in range(nrec):
            for k in names:
                out[k][g, tmin:tmax] *= rs[g]
                obs[k][g, tmin:tmax] *= rs0[g]
    else:
        rs[:] = 1
    rn = np.zeros(nrec)
    if scalerms or scalermsnorm:
        for g in range(nrec):
            acc = 0.0
            for k in names:
                for t in range(tmin, tmax):
                    acc += out[k][g, t] * (out[k][g, t] - obs[k][g, t])
            if scalerms:
                acc *= (ws / rs0[g] / ws) ** 2
            rn[g] = 1.0 - acc
    rms = rmsnorm = 0.0
    res = {k: np.zeros_like(out[k]) for k in names}
    for g in range(nrec):
        for t in range(tmax):
            for k in names:
                rms += (obs[k][g, t] - out[k][g, t]) ** 2
                rmsnorm += obs[k][g, t] ** 2
                if scalermsnorm or scalerms:
                    res[k][g, t] = rs[g] * ((1.0 - rn[g]) * out[k][g, t] - obs[k][g, t])
                else:
                    res[k][g, t] = rs[g] * (out[k][g, t] - obs[k][g, t])
    return res, rms, rmsnorm


@pytest.mark.parametrize("flags", [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1)])
def test_residuals_match_loop_restatement(flags):
    scalerms, scalermsnorm, scaleshot = flags
    s = _seis(NT=40, scalerms=scalerms, scalermsnorm=scalermsnorm, scaleshot=scaleshot, tmin=0.0055)
    rng = np.random.default_rng(1)
    out = {k: rng.standard_normal((5, 40)).astype(np.float32) for k in ("vx", "vz")}
    obs = {k: (0.8 * out[k] + 0.3 * rng.standard_normal((5, 40))).astype(np.float32) for k in out}
    tmax = 36
    res, rms, rmsnorm = s._residuals(out, obs, None, 40, tmax)
    want, wrms, wnorm = _residuals_loops(out, obs, 5, tmax, scalerms, scalermsnorm, scaleshot)
    for k in out:
        assert np.allclose(res[k], want[k], rtol=1e-5, atol=1e-6), k
        assert np.all(res[k][:, tmax:] == 0)
    assert np.isclose(rms, wrms, rtol=1e-5) and np.isclose(rmsnorm, wnorm, rtol=1e-5)


def test_dft_misfit_matches_direct_transform():
    """back_prop_type 2: the misfit is taken at the gradient frequencies only,
    |DFT|^2 of the residual and of the data at bin int(f*nfft*dt + 1) of a
    next_fast_size(tmax) transform (residuals.c:254-410); the adjoint sources
    stay those of the time domain."""
    from seiscl_b200.seiscl import next_fast_size

    freqs = np.array([90.0, 180.0, 333.0])
    s = _seis(NT=40, back_prop_type=2, gradfreqs=freqs)
    s1 = _seis(NT=40)
    rng = np.random.default_rng(4)
    out = {k: rng.standard_normal((5, 40)).astype(np.float32) for k in ("vx", "vz")}
    obs = {k: (0.8 * out[k] + 0.3 * rng.standard_normal((5, 40))).astype(np.float32) for k in out}
    tmax = 37
    res, rms, rmsnorm = s._residuals(out, obs, None, 40, tmax)
    res1, _, _ = s1._residuals(out, obs, None, 40, tmax)
    nfft = next_fast_size(tmax)
    want = wnorm = 0.0
    t = np.arange(tmax)
    for f in freqs:
        b = int(np.float32(f) * nfft * np.float32(s.dt) + 1)
        e = np.exp(-2j * np.pi * b * t / nfft)
        for k in out:
            for g in range(5):
                want += abs(np.sum((obs[k][g, :tmax].astype(np.float64) - out[k][g, :tmax]) * e)) ** 2
                wnorm += abs(np.sum(obs[k][g, :tmax].astype(np.float64) * e)) ** 2
    assert np.isclose(rms, want, rtol=1e-9) and np.isclose(rmsnorm, wnorm, rtol=1e-9)
    for k in out:
        assert np.array_equal(res[k], res1[k])


def test_dft_job_needs_frequencies():
    from seiscl_b200.seiscl import SeisCLError

    s = _seis(back_prop_type=2, gradout=1)
    with pytest.raises(SeisCLError):
        s._engine_config()
    s.gradfreqs = np.array([[5.0, 10.0]])
    c = s._engine_config()
    assert c.back_prop_type == 2 and c.gradfreqs == (5.0, 10.0)
    s.back_prop_type = 3
    with pytest.raises(SeisCLError):
        s._engine_config()


# ------------------------------------------------------------------ GPU jobs
def _two_shot_job(**kw):
    s = _seis(**kw)
    nz, nx = s.N
    zs = 6 * s.dh
    s.src_pos_all = np.array([[20 * s.dh, 38 * s.dh], [0, 0], [zs, zs], [0, 1], [100, 100]], float)
    xg = np.arange(13, nx - 13, 3) * s.dh
    rec = []
    for sid in (0, 1):
        r = np.zeros((8, len(xg)))
        r[0], r[2], r[3] = xg, zs + 4 * s.dh, sid
        rec.append(r)
    s.rec_pos_all = np.concatenate(rec, 1)
    s.rec_pos_all[4] = np.arange(1, s.rec_pos_all.shape[1] + 1)
    return s


def _oracle_cfg(s):
    nz, nx = (int(v) for v in s.N)
    return dict(nd=s.ND, nz=nz, nx=nx, ny=1, nt=s.NT, dt=s.dt, dh=s.dh, nab=s.nab, freesurf=s.freesurf,
                L=s.L, abs_type=s.abs_type, fdorder=s.FDORDER, f0=s.f0, fl=[15.0])


def _oracle_for(s, model):
    from oracle.oracle import Oracle

    o = Oracle(_oracle_cfg(s))
    assert o.set_model(model["vp"].T, model["vs"].T, model["rho"].T) == 0
    return o


def _shot_rows(s, sid):
    sp = s.src_pos_all.T.astype(np.float32)
    rp = s.rec_pos_all.T.astype(np.float32)
    src = np.stack([ricker(s.f0, s.NT, s.dt)] * len(sp))
    si = sp[:, 3] == sid
    gi = rp[:, 3] == sid
    return sp[si], src[si], rp[gi], gi


@pytest.mark.gpu
def test_forward_job_matches_oracle(cuda_device):
    s = _two_shot_job()
    model = _models(tuple(s.N), 5)
    s.set_forward(s.src_pos_all[3, :], model, withgrad=False)
    s.execute()
    vx, vz = s.read_data()
    assert vx.shape == (s.NT, s.rec_pos_all.shape[1])
    o = _oracle_for(s, model)
    for sid in (0, 1):
        sp, src, rp, gi = _shot_rows(s, sid)
        d = o.forward(sp, src, rp, ["vx", "vz"])
        assert rel_l2(vx[:, gi].T, d["vx"]) < FWD_TOL
        assert rel_l2(vz[:, gi].T, d["vz"]) < FWD_TOL


@pytest.mark.gpu
def test_gradient_job_matches_oracle(cuda_device):
    s = _two_shot_job(rmsout=1)
    true = _models(tuple(s.N), 7)
    start = _models(tuple(s.N), 8)
    o_true = _oracle_for(s, true)
    obs = {}
    for sid in (0, 1):
        sp, src, rp, gi = _shot_rows(s, sid)
        obs[sid] = o_true.forward(sp, src, rp, ["vx", "vz"])
    data = {k: np.concatenate([obs[0][k], obs[1][k]], 0).T for k in ("vx", "vz")}
    s.prepare_data(s.src_pos_all[3, :])
    s.write_data(data)
    s.cropgrad = False
    s.set_forward(s.src_pos_all[3, :], start, withgrad=True)
    s.execute()
    gvp, gvs, grho = s.read_grad()
    rms, rms_norm = s.read_rms()

    o = _oracle_for(s, start)
    o.clear_gradients()
    r2 = n2 = 0.0
    for sid in (0, 1):
        sp, src, rp, gi = _shot_rows(s, sid)
        d = o.forward(sp, src, rp, ["vx", "vz"], save_boundaries=True)
        res = {k: d[k] - obs[sid][k] for k in d}
        r2 += sum(float(((obs[sid][k].astype(np.float64) - d[k]) ** 2).sum()) for k in d)
        n2 += sum(float((obs[sid][k].astype(np.float64) ** 2).sum()) for k in d)
        o.adjoint(sp, src, rp, o.residual_scale(rp, res))
    g = o.gradients()
    for name, got in (("vp", gvp), ("vs", gvs), ("rho", grho)):
        assert np.abs(g[name]).max() > 0
        assert rel_l2(got.T, g[name]) < GRAD_TOL, name
    assert np.isclose(rms_norm, np.sqrt(n2), rtol=1e-4)
    assert np.isclose(rms, np.sqrt(r2) / np.sqrt(n2), rtol=1e-3)


@pytest.mark.gpu
def test_inputres_job_equals_combined_job(cuda_device):
    """set_backward(residuals) after a forward run gives the gradient of a
    single run that computes the same residuals itself."""
    s = _two_shot_job()
    model = _models(tuple(s.N), 9)
    s.set_forward(s.src_pos_all[3, :], model, withgrad=False)
    s.execute()
    d = s.read_data()
    obs = {"vx": (0.7 * d[0]).astype(np.float32), "vz": (0.7 * d[1]).astype(np.float32)}
    s.write_data(obs)
    s.cropgrad = False
    s.set_forward(s.src_pos_all[3, :], model, withgrad=True)
    s.execute()
    g_comb = s.read_grad()
    s.inputres = 1
    s.set_forward(s.src_pos_all[3, :], model, withgrad=False)
    s.set_backward(residuals=[d[0] - obs["vx"], d[1] - obs["vz"]])
    s.execute()
    g_in = s.read_grad()
    for a, b in zip(g_in, g_comb):
        assert rel_l2(a, b) < 1e-6


@pytest.mark.gpu
def test_dft_gradient_job_matches_oracle(cuda_device):
    """A two-shot DFT-gradient job (back_prop_type 2) through the front end
    against the oracle driven the same way; the misfit at the gradient
    frequencies from the oracle's seismograms."""
    from seiscl_b200.seiscl import next_fast_size

    freqs = np.array([9.0, 17.0, 26.0])
    s = _two_shot_job(rmsout=1, back_prop_type=2, gradfreqs=freqs)
    true = _models(tuple(s.N), 17)
    start = _models(tuple(s.N), 18)
    o_true = _oracle_for(s, true)
    obs = {}
    for sid in (0, 1):
        sp, src, rp, gi = _shot_rows(s, sid)
        obs[sid] = o_true.forward(sp, src, rp, ["vx", "vz"])
    data = {k: np.concatenate([obs[0][k], obs[1][k]], 0).T for k in ("vx", "vz")}
    s.prepare_data(s.src_pos_all[3, :])
    s.write_data(data)
    s.cropgrad = False
    s.set_forward(s.src_pos_all[3, :], start, withgrad=True)
    s.execute()
    gvp, gvs, grho = s.read_grad()
    rms, rms_norm = s.read_rms()

    from oracle.oracle import Oracle

    cfg = _oracle_cfg(s)
    cfg.update(back_prop_type=2, gradfreqs=list(freqs))
    o = Oracle(cfg)
    assert o.set_model(start["vp"].T, start["vs"].T, start["rho"].T) == 0
    o.clear_gradients()
    nfft = next_fast_size(s.NT)
    bins = [int(np.float32(f) * nfft * np.float32(s.dt) + 1) for f in freqs]
    r2 = n2 = 0.0
    for sid in (0, 1):
        sp, src, rp, gi = _shot_rows(s, sid)
        d = o.forward(sp, src, rp, ["vx", "vz"], save_boundaries=True)
        res = {k: d[k] - obs[sid][k] for k in d}
        for k in d:
            r2 += float((np.abs(np.fft.rfft(obs[sid][k].astype(np.float64) - d[k], n=nfft)[:, bins]) ** 2).sum())
            n2 += float((np.abs(np.fft.rfft(obs[sid][k].astype(np.float64), n=nfft)[:, bins]) ** 2).sum())
        o.adjoint(sp, src, rp, o.residual_scale(rp, res))
    g = o.raw_gradients()
    for name, got in (("M", gvp), ("mu", gvs), ("rho", grho)):
        assert np.abs(g[name]).max() > 0
        assert rel_l2(got.T, g[name]) < GRAD_TOL, name
    assert np.isclose(rms_norm, np.sqrt(n2), rtol=1e-4)
    assert np.isclose(rms, np.sqrt(r2) / np.sqrt(n2), rtol=1e-3)


@pytest.mark.gpu
def test_hessian_job_returns_the_engine_hessian(cuda_device):
    """Hout=1: read_Hessian returns the engine's transformed Hessian summed
    over the job's shots, cropped like read_grad."""
    s = _two_shot_job(Hout=1)
    model = _models(tuple(s.N), 11)
    s.set_forward(s.src_pos_all[3, :], model, withgrad=False)
    s.execute()
    d = s.read_data()
    s.write_data({"vx": (0.7 * d[0]).astype(np.float32), "vz": (0.7 * d[1]).astype(np.float32)})
    s.cropgrad = False
    s.set_forward(s.src_pos_all[3, :], model, withgrad=True)
    s.execute()
    H = s.read_Hessian()
    assert len(H) == 3 and H[0].shape == tuple(s.N)
    assert np.abs(H[0]).max() > 0 and np.abs(H[1]).max() > 0
    s.cropgrad = True
    Hc = s.read_Hessian()
    assert np.all(Hc[0][:, :s.nab] == 0) and np.array_equal(Hc[0][30, 30], H[0][30, 30])
