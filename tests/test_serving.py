"""The modelling service (seiscl_b200.serving).

CPU: scheduling, error reporting and result independence with a
deterministic stand-in for the engine.  GPU: concurrent requests on one B200
give bit-identical results to the same requests run one by one.
"""
import numpy as np
import pytest

from tests._cases import engine_config, make_case


class FakePlan:
    def __init__(self, cfg):
        self.cfg = cfg
        self.tmax = cfg.NT

    def close(self):
        pass

    def set_model(self, vp, vs, rho, taup=None, taus=None):
        self.m = float(np.mean(vp)) + 0.5 * float(np.mean(rho))

    def zero_gradient(self):
        self.g = 0.0

    def forward(self, sp, src, rp, outs, save_boundaries=False):
        t = np.arange(self.cfg.NT, dtype=np.float32)
        return {k: (np.cos(1e-3 * self.m * t) * (i + 1) * (1 + rp[:, :1] * 1e-3)).astype(np.float32)
                for i, k in enumerate(outs)}

    def residual_scale(self, rp, res):
        return res

    def adjoint(self, sp, src, rp, res):
        self.g += sum(float(v.sum()) for v in res.values())

    def gradient(self, transform=True):
        return {"vp": np.full((4, 4), self.g, np.float32)}


def _requests(n, seed=0):
    from seiscl_b200.engine import Config
    from seiscl_b200.serving import Request

    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nx, nz = int(rng.integers(30, 60)), int(rng.integers(30, 60))
        cfg = Config(N=[nz, nx], ND=2, NT=50, nab=8)
        m = {"vp": np.full((nx, nz), 3000.0 + 10 * i, np.float32), "vs": np.full((nx, nz), 1700.0, np.float32),
             "rho": np.full((nx, nz), 2000.0, np.float32)}
        shots = [(np.array([[100.0, 0, 100.0, 0, 100]], np.float32), np.zeros((1, 50), np.float32),
                  np.array([[150.0 + 10 * j, 0, 100.0, 0, j + 1, 0, 0, 0] for j in range(3)], np.float32))]
        kind = "gradient" if i % 3 == 0 else "forward"
        obs = [{"vx": np.zeros((3, 50), np.float32), "vz": np.zeros((3, 50), np.float32)}] if kind == "gradient" else None
        out.append(Request(cfg, m, shots, ("vx", "vz"), kind, obs, rid=i))
    return out


def test_server_results_equal_serial_runs(monkeypatch):
    from seiscl_b200 import engine, serving

    monkeypatch.setattr(engine, "Plan", FakePlan)
    reqs = _requests(12)
    with serving.Server(workers=3, plans_per_worker=2) as srv:
        futs = [srv.submit(r) for r in reqs]
        res = [f.result(timeout=60) for f in futs]
    for r, q in zip(res, reqs):
        ref = serving.serve(FakePlan(q.config), q)
        assert r.rid == q.rid and r.latency >= 0
        for a, b in zip(r.seismograms, ref.seismograms):
            for k in a:
                assert np.array_equal(a[k], b[k])
        if q.kind == "gradient":
            assert np.array_equal(r.gradient["vp"], ref.gradient["vp"]) and r.misfit == ref.misfit
    p = serving.percentiles([r.latency for r in res])
    assert p["p50"] <= p["p99"]


def test_server_reports_errors_through_futures(monkeypatch):
    from seiscl_b200 import engine, serving

    monkeypatch.setattr(engine, "Plan", FakePlan)
    bad = _requests(1)[0]
    bad.kind = "nonsense"
    with serving.Server(workers=1) as srv:
        f = srv.submit(bad)
        with pytest.raises(ValueError):
            f.result(timeout=60)
        ok = srv.submit(_requests(2)[1]).result(timeout=60)
        assert ok.rid == 1
    with pytest.raises(RuntimeError):
        srv.submit(bad)


@pytest.mark.gpu
def test_concurrent_requests_are_deterministic(cuda_device):
    from seiscl_b200 import serving
    from seiscl_b200.engine import Plan

    reqs = []
    for i, kw in enumerate([dict(nd=2, freesurf=1, L=0, seed=1), dict(nd=2, freesurf=0, L=1, seed=2),
                            dict(nd=2, freesurf=1, L=0, seed=3, nz=64, nx=40), dict(nd=2, freesurf=0, L=0, seed=4)]):
        cfg, model, acq = make_case(**kw)
        shots = [(acq["src_pos"], acq["src"], acq["rec_pos"])]
        kind = "gradient" if i % 2 else "forward"
        obs = None
        if kind == "gradient":
            obs = [{"vx": np.zeros((len(acq["rec_pos"]), cfg["nt"]), np.float32),
                    "vz": np.zeros((len(acq["rec_pos"]), cfg["nt"]), np.float32)}]
        m = {k: v for k, v in model.items() if v is not None}
        reqs.append(serving.Request(engine_config(cfg), m, shots, ("vx", "vz"), kind, obs, rid=i))
    serial = []
    for q in reqs:
        p = Plan(q.config)
        serial.append(serving.serve(p, q))
        p.close()
    with serving.Server(workers=4) as srv:
        futs = [srv.submit(q) for q in reqs * 3]
        res = [f.result(timeout=300) for f in futs]
    for i, r in enumerate(res):
        ref = serial[i % len(reqs)]
        for a, b in zip(r.seismograms, ref.seismograms):
            for k in a:
                assert np.array_equal(a[k], b[k]), (i, k)
        if ref.gradient is not None:
            for k in ref.gradient:
                assert np.array_equal(r.gradient[k], ref.gradient[k]), (i, k)
