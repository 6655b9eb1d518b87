"""The modelling service (seiscl_b200.serving).

CPU: scheduling, error reporting and result independence with a
deterministic stand-in for the engine.  GPU: concurrent requests on one B200
give bit-identical results to the same requests run one by one.
"""
import dataclasses

import numpy as np
import pytest

from tests._cases import engine_config, make_case, rel_l2


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

    def forward_batch(self, shots, outs, save_boundaries=False):
        assert len(shots) <= self.cfg.batch
        return [self.forward(sp, src, rp, outs, save_boundaries) for sp, src, rp in shots]

    def adjoint_batch(self, shots, residuals):
        for (sp, src, rp), r in zip(shots, residuals):
            self.adjoint(sp, src, rp, r)


def _requests(n, seed=0):
    from seiscl_b200.engine import Config
    from seiscl_b200.serving import Request

    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nx, nz = int(rng.integers(30, 60)), int(rng.integers(15, 30)) * 2
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
    with serving.Server(workers=3, plans_per_worker=2, memory_budget=1 << 40) as srv:
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
    with serving.Server(workers=1, memory_budget=1 << 40) as srv:
        f = srv.submit(bad)
        with pytest.raises(ValueError):
            f.result(timeout=60)
        ok = srv.submit(_requests(2)[1]).result(timeout=60)
        assert ok.rid == 1
    with pytest.raises(RuntimeError):
        srv.submit(bad)


class CountingPlan(FakePlan):
    """FakePlan that records how many plans are alive and holds the GPU for
    a while, so that requests overlap."""
    alive = 0
    peak = 0
    lock = None

    def __init__(self, cfg):
        super().__init__(cfg)
        with CountingPlan.lock:
            CountingPlan.alive += 1
            CountingPlan.peak = max(CountingPlan.peak, CountingPlan.alive)

    def close(self):
        with CountingPlan.lock:
            CountingPlan.alive -= 1

    def forward(self, *a, **k):
        import time

        time.sleep(0.01)
        return super().forward(*a, **k)


def _fake_footprint(req):
    """Bytes proportional to the grid (any positive measure will do)."""
    return int(np.prod(req.config.N)) * (3 if req.kind == "gradient" else 1)


def test_admission_keeps_held_memory_within_budget(monkeypatch):
    """Every admitted plan counts at its footprint; with a budget of about
    two requests, never more than the budget is held, idle plans are evicted
    to admit new configurations, and results are unchanged."""
    import threading

    from seiscl_b200 import engine, serving

    CountingPlan.alive = CountingPlan.peak = 0
    CountingPlan.lock = threading.Lock()
    monkeypatch.setattr(engine, "Plan", CountingPlan)
    reqs = _requests(16, seed=3)
    sizes = [_fake_footprint(q) for q in reqs]
    budget = 2 * max(sizes)
    with serving.Server(workers=4, plans_per_worker=2, memory_budget=budget, footprint=_fake_footprint) as srv:
        res = [f.result(timeout=60) for f in [srv.submit(q) for q in reqs]]
        st = srv.stats()
    assert st["peak_bytes"] <= budget and st["admitted"] == len(reqs) and st["rejected"] == 0
    assert st["evicted"] > 0
    assert CountingPlan.alive == 0           # every plan closed at the end
    for r, q in zip(res, reqs):
        ref = serving.serve(FakePlan(q.config), q)
        for a, b in zip(r.seismograms, ref.seismograms):
            for k in a:
                assert np.array_equal(a[k], b[k])


def test_admission_rejects_requests_larger_than_the_budget(monkeypatch):
    from seiscl_b200 import engine, serving

    monkeypatch.setattr(engine, "Plan", FakePlan)
    reqs = _requests(4, seed=4)
    big = max(reqs, key=_fake_footprint)
    budget = _fake_footprint(big) - 1
    with serving.Server(workers=2, memory_budget=budget, footprint=_fake_footprint) as srv:
        futs = [srv.submit(q) for q in reqs]
        for q, f in zip(reqs, futs):
            if q is big:
                with pytest.raises(MemoryError):
                    f.result(timeout=60)
            else:
                assert f.result(timeout=60).rid == q.rid
        assert srv.stats()["rejected"] == 1


def _multi_shot_request(nd, nshots, seed):
    from seiscl_b200 import serving

    q = _requests(1, seed=seed)[0]
    if nd == 3:   # FP16 wave fields: not batched
        q.config = dataclasses.replace(q.config, ND=3, N=[20, 20, 20], field_precision="fp16")
    sp, src, rp = q.shots[0]
    q.shots = [(sp, src, rp + np.float32(j)) for j in range(nshots)]
    q.kind = "gradient"
    q.observed = [{"vx": np.full((3, 50), 0.1 * j, np.float32), "vz": np.zeros((3, 50), np.float32)}
                  for j in range(nshots)]
    return q


@pytest.mark.parametrize("nd", [2, 3])
def test_batches_and_slots_keep_shot_order_and_sum_gradients(monkeypatch, nd):
    """2D requests advance their shots in batches on one plan; others may
    spread them over plans running at once (shot i on plan i % k).
    Seismograms come back in shot order and gradients are summed in a fixed
    order, so the service and ``serve_alone`` agree exactly."""
    from seiscl_b200 import engine, serving

    monkeypatch.setattr(engine, "Plan", FakePlan)
    q = _multi_shot_request(nd, 6, seed=6)
    fp = lambda r: 1000
    cfg = serving.plan_config(q)
    assert cfg.batch == (6 if nd == 2 else 1)
    slots = serving.shot_slots(q, fp(q), max_slots=4)
    assert slots == (1 if nd == 2 else 4)
    alone = serving.serve_alone(q, max_slots=4, footprint=fp)
    with serving.Server(workers=2, memory_budget=1 << 20, footprint=fp, max_slots=4) as srv:
        got = srv.submit(q).result(timeout=60)
        assert srv.stats()["slots"] == slots
    one = serving.serve(FakePlan(q.config), q)
    for i in range(6):
        for k in ("vx", "vz"):
            assert np.array_equal(got.seismograms[i][k], alone.seismograms[i][k])
            assert np.array_equal(got.seismograms[i][k], one.seismograms[i][k])
    assert np.array_equal(got.gradient["vp"], alone.gradient["vp"]) and got.misfit == alone.misfit
    assert np.allclose(got.gradient["vp"], one.gradient["vp"], rtol=1e-6) and got.misfit == one.misfit


def test_router_spreads_requests_over_servers(monkeypatch):
    """One server per device; each request goes to the least busy one and
    comes back unchanged."""
    import threading

    from seiscl_b200 import engine, serving

    CountingPlan.alive = CountingPlan.peak = 0
    CountingPlan.lock = threading.Lock()
    monkeypatch.setattr(engine, "Plan", CountingPlan)
    reqs = _requests(12, seed=8)
    with serving.Router([None, None, None], workers=1, memory_budget=1 << 40,
                        footprint=_fake_footprint) as router:
        res = [f.result(timeout=60) for f in [router.submit(q) for q in reqs]]
        admitted = [st["admitted"] for st in router.stats()]
    assert sum(admitted) == len(reqs) and min(admitted) >= 1
    for r, q in zip(res, reqs):
        ref = serving.serve(FakePlan(q.config), q)
        assert r.rid == q.rid
        for a, b in zip(r.seismograms, ref.seismograms):
            for k in a:
                assert np.array_equal(a[k], b[k])


def test_footprint_grows_with_grid_and_gradient_buffers():
    from seiscl_b200 import engine

    c2 = engine.Config(N=[200, 300], ND=2, NT=1000, nab=16)
    f2 = engine.footprint(c2, False, 1, 200)
    g2 = engine.footprint(c2, True, 1, 200)
    # wave fields, parameters and seismograms alone: 5 + 14 arrays of the grid
    assert f2 >= 4 * (5 * 208 * 308 + 14 * 200 * 300) + 4 * 2 * 200 * 1000
    assert g2 > f2
    c3 = engine.Config(N=[64, 64, 64], ND=3, NT=500, L=2, FL=[5.0, 40.0], nab=10)
    f3 = engine.footprint(c3, False, 1, 100)
    assert f3 > engine.footprint(engine.Config(N=[64, 64, 64], ND=3, NT=500, nab=10), False, 1, 100)
    import dataclasses
    h3 = engine.footprint(dataclasses.replace(c3, precision="fp16"), True, 1, 100)
    assert engine.footprint(c3, True, 1, 100) > h3 > f3


@pytest.mark.gpu
def test_footprint_matches_device_allocation(cuda_device):
    """The footprint computed from the configuration equals what a plan
    allocates for forward and gradient runs (2D, 3D, viscoelastic, FP16
    boundaries, DFT gradient)."""
    import dataclasses

    from seiscl_b200 import engine
    from seiscl_b200.engine import Plan

    cases = [(dict(nd=2, nz=200, nx=300, nt=400, nab=16), {}),
             (dict(nd=3, nz=64, ny=60, nx=68, nt=200, nab=10, L=2), {}),
             (dict(nd=2, nz=80, nx=90, nt=300, nab=12, L=1), dict(precision="fp16")),
             (dict(nd=2, nz=80, nx=90, nt=300, nab=12, L=1), dict(back_prop_type=2, gradfreqs=[5.0, 10.0, 15.0]))]
    for kw, extra in cases:
        cfg, model, acq = make_case(**kw)
        ec = dataclasses.replace(engine_config(cfg), **extra)
        nrec = len(acq["rec_pos"])
        for grad in (False, True):
            plan = Plan(ec)
            if ec.back_prop_type == 2:
                plan.set_gradfreqs(ec.gradfreqs)
            plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
            d = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], ["vx", "vz"], save_boundaries=grad)
            if grad:
                plan.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], d)
            got = plan.device_bytes
            plan.close()
            est = engine.footprint(ec, grad, 1, nrec * 2, len(ec.gradfreqs))
            assert got == est, (kw, extra, grad, est, got)


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
    # requests whose five shots advance together in one batched plan
    cfg, model, acq = make_case(nd=2, freesurf=1, L=0, seed=5)
    shots = [(acq["src_pos"] + np.array([[10.0 * j, 0, 0, j, 0]], np.float32), acq["src"], acq["rec_pos"])
             for j in range(5)]
    obs = [{"vx": np.zeros((len(acq["rec_pos"]), cfg["nt"]), np.float32),
            "vz": np.zeros((len(acq["rec_pos"]), cfg["nt"]), np.float32)} for _ in shots]
    m = {k: v for k, v in model.items() if v is not None}
    reqs.append(serving.Request(engine_config(cfg), m, shots, ("vx", "vz"), "gradient", obs, rid=len(reqs)))
    reqs.append(serving.Request(engine_config(cfg), m, shots, ("vx", "vz"), "forward", None, rid=len(reqs)))
    assert serving.plan_config(reqs[-1]).batch == 5 and serving.plan_config(reqs[-2]).batch == 5
    serial = [serving.serve_alone(q) for q in reqs]
    # one plan, shots one after another: the same seismograms, the gradient to rounding
    one = serving.serve(Plan(reqs[-2].config), reqs[-2])
    for a, b in zip(one.seismograms, serial[-2].seismograms):
        for k in a:
            assert np.array_equal(a[k], b[k]), k
    for k in one.gradient:
        assert rel_l2(one.gradient[k], serial[-2].gradient[k]) < 1e-6, k
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


def _grad_request(cfg, model, acq, nshots=3):
    from seiscl_b200.serving import Request

    shots = [(acq["src_pos"], acq["src"], acq["rec_pos"])] * nshots
    nrec, nt = acq["rec_pos"].shape[0], cfg.NT
    obs = [{"vx": np.zeros((nrec, nt), np.float32), "vz": np.zeros((nrec, nt), np.float32)} for _ in shots]
    return Request(cfg, model, shots, ("vx", "vz"), "gradient", obs)


def test_viscoelastic_gradient_requests_recompute_from_snapshots():
    """Gradient requests with memory variables run the snapshot-checkpoint
    recompute, one shot per launch (the reference's backpropagation of
    memory variables is unstable over long runs); elastic ones batch."""
    from seiscl_b200.serving import CHECKPOINT_STEPS, plan_config

    cfg, model, acq = make_case(nd=2, L=2, nt=60, seed=8)
    c = plan_config(_grad_request(engine_config(cfg), model, acq))
    assert c.checkpoint == CHECKPOINT_STEPS and c.batch in (0, 1)
    cfg, model, acq = make_case(nd=2, L=0, nt=60, seed=8)
    c = plan_config(_grad_request(engine_config(cfg), model, acq))
    assert not c.checkpoint and c.batch == 3


@pytest.mark.gpu
def test_viscoelastic_gradient_request_stays_finite(cuda_device):
    """A 2D viscoelastic gradient request of 1200 steps through the service:
    finite gradients (the boundary-saving backpropagation of the memory
    variables can overflow on runs this long)."""
    from seiscl_b200.serving import serve_alone

    cfg, model, acq = make_case(nd=2, L=2, nt=1200, nz=60, nx=80, nab=10, seed=9)
    r = serve_alone(_grad_request(engine_config(cfg), model, acq, nshots=2))
    assert set(r.gradient) >= {"vp", "vs", "rho"}
    for k, v in r.gradient.items():
        assert np.isfinite(v).all(), k
        assert np.abs(v).max() > 0, k


@pytest.mark.gpu
def test_acoustic_gradients(cuda_device):
    """Acoustic media (P-SV with vs = 0): with a free surface the adjoint is
    refused with a message (the free-surface adjoint divides by mu); without
    one the service returns finite vp and rho gradients and no vs gradient."""
    from seiscl_b200.engine import Plan, SeisCLEngineError
    from seiscl_b200.serving import serve_alone

    cfg, model, acq = make_case(nd=2, L=0, nt=150, seed=10)
    model = dict(model, vs=np.zeros_like(model["vs"]))
    plan = Plan(engine_config(cfg))
    plan.set_model(model["vp"], model["vs"], model["rho"])
    d = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], ["vx", "vz"], save_boundaries=True)
    with pytest.raises(SeisCLEngineError, match="free-surface adjoint"):
        plan.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], d)
    plan.close()
    cfg0 = dataclasses.replace(engine_config(cfg), freesurf=0)
    r = serve_alone(_grad_request(cfg0, model, acq, nshots=2))
    assert "vs" not in r.gradient
    for k in ("vp", "rho"):
        assert np.isfinite(r.gradient[k]).all() and np.abs(r.gradient[k]).max() > 0, k
