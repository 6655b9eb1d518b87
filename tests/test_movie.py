"""Movie output (SeisCL's MOVOUT, src/time_stepping.c:272-350).

Every `movout` steps the physical cells of each recorded wave field are
copied to a snapshot.  Checked against the oracle: snapshot m - 1 of a run
equals the oracle's field after a run stopped at step m * movout (forward),
and, for a boundary-saving gradient, the reconstructed forward field after
an adjoint stopped at the snapshot's step.  The front end returns the
movie in the reference's orientation.
"""
import numpy as np
import pytest

from tests._cases import engine_config, make_case, rel_l2

TOL = 2e-5


def _interior(o, name, cfg):
    F = cfg["fdorder"] // 2
    a = o.array("wave", name)
    if cfg["nd"] == 3:
        a = a.reshape(o.NXp, o.NYp, o.NZp)[F:-F, F:-F, F:-F]
    else:
        a = a.reshape(o.NXp, o.NZp)[F:-F, F:-F]
    return a


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(nd=2, freesurf=1, L=1, abs_type=1, src_type=100, nt=120, seed=41),
                                dict(nd=3, freesurf=1, L=0, abs_type=1, src_type=2, nz=36, ny=30, nx=34, nt=60,
                                     nab=8, seed=42)],
                         ids=["2d", "3d"])
def test_forward_movie_matches_oracle_fields(kw, cuda_device):
    from oracle.oracle import Oracle
    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(**kw)
    movout = 20
    names = ["vx", "vz", "sxx", "szz", "sxz"] + (["vy", "syy", "sxy", "syz"] if cfg["nd"] == 3 else [])
    plan = Plan(engine_config(cfg))
    plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    mov = plan.set_movie(movout, names)
    plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], names)
    nslot = cfg["nt"] // movout
    assert all(m.shape[0] == nslot for m in mov.values())
    for m in (1, nslot // 2, nslot):
        c = dict(cfg, tmax=m * movout)
        o = Oracle(c)
        o.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
        o.forward(acq["src_pos"], acq["src"], acq["rec_pos"], ["vx"])
        for n in names:
            ref = _interior(o, n, cfg)
            assert np.abs(ref).max() > 0, (m, n)
            assert rel_l2(mov[n][m - 1], ref) < TOL, (m, n, rel_l2(mov[n][m - 1], ref))
    plan.set_movie(0)


@pytest.mark.gpu
def test_gradient_movie_films_the_reconstruction(cuda_device):
    """Boundary-saving gradient: the forward run films nothing; the adjoint
    films the reconstructed forward field after step t (t % movout == 0)
    into snapshot (t + 1) // movout - 1."""
    from oracle.oracle import Oracle
    from seiscl_b200.engine import Plan

    cfg, model, acq = make_case(nd=2, freesurf=0, L=0, abs_type=1, src_type=100, nt=120, seed=43)
    movout = 20
    names = ["vx", "vz"]
    plan = Plan(engine_config(cfg))
    plan.set_model(model["vp"], model["vs"], model["rho"])
    mov = plan.set_movie(movout, names)
    d = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], names, save_boundaries=True)
    assert all(np.abs(m).max() == 0 for m in mov.values())
    res = {k: (0.3 * v).astype(np.float32) for k, v in d.items()}
    plan.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], res)
    for t in (40, 100):
        slot = (t + 1) // movout - 1
        o = Oracle(dict(cfg, tmin=t - 1))
        o.set_model(model["vp"], model["vs"], model["rho"])
        o.forward(acq["src_pos"], acq["src"], acq["rec_pos"], names, save_boundaries=True)
        o.adjoint(acq["src_pos"], acq["src"], acq["rec_pos"], res)
        for n in names:
            ref = _interior(o, n, cfg)
            assert rel_l2(mov[n][slot], ref) < 5e-4, (t, n, rel_l2(mov[n][slot], ref))
    # snapshot 5 (t = 120) lies beyond the adjoint's first step (t = 119): empty
    assert np.abs(mov["vx"][5]).max() == 0 and np.abs(mov["vx"][0]).max() > 0
    plan.set_movie(0)


@pytest.mark.gpu
def test_front_end_movie_orientation(cuda_device):
    from seiscl_b200.engine import Plan
    from seiscl_b200.seiscl import SeisCL

    s = SeisCL(ND=2, N=np.array([48, 60]), dh=10.0, dt=1e-3, NT=100, nab=10, freesurf=1, f0=15.0, seisout=1,
               movout=25, workdir="unused")
    s.src_pos_all = np.array([[200.0, 300.0], [0, 0], [60.0, 60.0], [0, 1], [100, 100]])
    s.rec_pos_all = np.array([[300.0, 350.0], [0, 0], [60.0, 60.0], [0, 1], [1, 2], [0, 0], [0, 0], [0, 0]])
    rng = np.random.default_rng(5)
    vp = (3000 * (1 + 0.05 * rng.uniform(-1, 1, (48, 60)))).astype(np.float32)
    model = {"vp": vp, "vs": (vp / 1.8).astype(np.float32), "rho": np.full((48, 60), 2000.0, np.float32)}
    s.set_forward(s.src_pos_all[3], model, withgrad=False)
    s.execute()
    vx, vz = s.read_movie()
    assert vx.shape == (48, 60, 4, 2)
    plan = Plan(s._engine_config())
    plan.set_model(model["vp"].T, model["vs"].T, model["rho"].T)
    sp = s.src_pos_all.T.astype(np.float32)
    rp = s.rec_pos_all.T.astype(np.float32)
    src = s.src_all.T.astype(np.float32)
    for shot in (0, 1):
        mov = plan.set_movie(25, ["vx", "vz"])
        plan.forward(sp[shot:shot + 1], src[shot:shot + 1], rp[shot:shot + 1], ["vx", "vz"])
        assert np.array_equal(np.transpose(vx[..., shot]), mov["vx"])
        assert np.array_equal(np.transpose(vz[..., shot]), mov["vz"])
    plan.set_movie(0)
