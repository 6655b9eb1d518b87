"""Shot sharding over ranks (seiscl_b200.shots) on CPU with gloo.

The split follows src/time_stepping.c:705-722 and the reductions
src/Out_MPI.c:70-160.  The engine is replaced by a deterministic CPU fake so
the world-size-2 run exercises the host orchestration of SeisCL.execute
without a GPU; the parity of the engine itself is covered by the GPU tests.
"""
import os
import socket

import numpy as np
import pytest


def _ref_split(ns, ngroup, gid):
    # loop restatement of time_stepping.c:705-722
    smin = 0
    for i in range(gid):
        smin += ns // ngroup + 1 if i < ns % ngroup else ns // ngroup
    smax = smin + (ns // ngroup + 1 if gid < ns % ngroup else ns // ngroup)
    return smin, smax


@pytest.mark.parametrize("ns,world", [(1, 1), (5, 2), (7, 3), (2, 4), (16, 8), (9, 4)])
def test_shot_range_matches_reference_split(ns, world):
    from seiscl_b200.shots import shot_range

    seen = []
    for r in range(world):
        a, b = shot_range(ns, r, world)
        assert (a, b) == _ref_split(ns, world, r)
        seen.extend(range(a, b))
    assert seen == list(range(ns))


class FakePlan:
    """Stands in for engine.Plan: seismograms and gradients are fixed
    functions of the shot, so sums over any split are predictable."""

    def __init__(self, cfg):
        self.cfg = cfg
        self.tmax = cfg.NT
        self.g = None

    def close(self):
        pass

    def set_model(self, *a):
        self.shape = np.asarray(a[2]).shape

    def zero_gradient(self):
        self.g = {k: np.zeros(self.shape, np.float32) for k in ("vp", "vs", "rho")}

    def forward(self, sp, src, rp, outs, save_boundaries=False):
        t = np.arange(self.cfg.NT, dtype=np.float32)
        return {k: (np.sin(0.01 * t * (1 + rp[:, 4:5])) * (1 + i) + sp[0, 0] * 1e-3).astype(np.float32)
                for i, k in enumerate(outs)}

    def residual_scale(self, rp, res):
        return {k: v * 0.5 for k, v in res.items()}

    def adjoint(self, sp, src, rp, res):
        s = sum(float(np.abs(v).sum()) for v in res.values())
        for i, k in enumerate(self.g):
            self.g[k] += np.float32(s * (i + 1) * 1e-3) + np.float32(sp[0, 0] * 1e-4)

    def gradient(self, transform=True):
        return {k: v.copy() for k, v in self.g.items()}


def _job():
    from seiscl_b200.seiscl import SeisCL

    s = SeisCL(ND=2, N=np.array([40, 50]), dh=10.0, dt=1e-3, NT=60, nab=8, seisout=1, workdir="unused",
               rmsout=1, resout=1)
    s.src_pos_all = np.array([[100.0, 150, 200, 250, 300], [0] * 5, [50.0] * 5, [0, 1, 2, 3, 4], [100] * 5])
    rec = []
    for sid in range(5):
        r = np.zeros((8, 6))
        r[0] = np.arange(6) * 40.0 + 60
        r[2] = 90.0
        r[3] = sid
        rec.append(r)
    s.rec_pos_all = np.concatenate(rec, 1)
    s.rec_pos_all[4] = np.arange(1, 31)
    model = {"vp": np.full((40, 50), 3000.0, np.float32), "vs": np.full((40, 50), 1700.0, np.float32),
             "rho": np.full((40, 50), 2000.0, np.float32)}
    s.prepare_data(s.src_pos_all[3])
    obs = {"vx": np.full((60, 30), 0.1, np.float32), "vz": np.full((60, 30), -0.2, np.float32)}
    s.write_data(obs)
    s.cropgrad = False
    s.set_forward(s.src_pos_all[3], model, withgrad=True)
    s.execute()
    return s.read_data(), s.read_data(residuals=True), s.read_grad(), s.read_rms()


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist

    from seiscl_b200 import engine

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    engine.Plan = FakePlan
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        data, res, grad, rms = _job()
        np.savez(os.path.join(out_dir, "r%d.npz" % rank), d0=data[0], d1=data[1], r0=res[0], r1=res[1],
                 g0=grad[0], g1=grad[1], g2=grad[2], rms=np.array(rms))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def test_two_rank_job_equals_single_process(tmp_path, monkeypatch):
    import torch.multiprocessing as mp

    from seiscl_b200 import engine

    monkeypatch.setattr(engine, "Plan", FakePlan)
    data, res, grad, rms = _job()
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        z = np.load(tmp_path / ("r%d.npz" % r))
        assert np.allclose(z["d0"], data[0]) and np.allclose(z["d1"], data[1])
        assert np.allclose(z["r0"], res[0]) and np.allclose(z["r1"], res[1])
        for i in range(3):
            assert np.allclose(z["g%d" % i], grad[i], rtol=1e-6)
        assert np.allclose(z["rms"], np.array(rms), rtol=1e-6)
