"""Shot lanes of reference-mode calls (efwi_set_lanes): 1, 2 and 3 lanes
give the same misfit bits, the same per-shot adjoint sources and scratch
traces, images equal up to the order of the per-shot sums, and the same
stencil launch counts."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _ready():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _problem():
    from efwi.engine import Grid, Shot
    from efwi import synthetic
    nz, nx, ny, np_, nt = 24, 36, 32, 5, 140
    g = Grid(nz, nx, ny, np_, nt, 10.0, 10.0, 10.0, 1e-3, 12.0)
    rng = np.random.default_rng(11)
    mz, mx, my = nz - 2 * np_, nx - 2 * np_, ny - 2 * np_
    vp = (2300.0 + 200.0 * rng.random((mz, mx, my))).astype(np.float32)
    vs = (vp / 1.732).astype(np.float32)
    rho = (310.0 * vp ** 0.25).astype(np.float32)
    true = synthetic.elastic_params(vp, vs, rho, np_)
    vp0 = np.full_like(vp, float(vp.mean()))
    init = synthetic.elastic_params(vp0, (vp0 / 1.732).astype(np.float32),
                                    (310.0 * vp0 ** 0.25).astype(np.float32), np_)
    xs = np.arange(np_, nx - np_, 3)
    ys = np.arange(np_, ny - np_, 3)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    zr = np.full(X.size, np_ + 1, np.int32)
    shots = [Shot(src=(np_ + 2, 8 + 4 * k, 9 + 3 * k), z_rec=zr, x_rec=X.ravel().astype(np.int32),
                  y_rec=Y.ravel().astype(np.int32)) for k in range(5)]
    stf = np.stack([synthetic.ricker(12.0, nt, 1e-3) for _ in range(5)])
    return g, shots, stf, true, init


def test_lanes_match_one_lane():
    from efwi.engine import Propagator
    g, shots, stf, true, init = _problem()
    ids = [0, 1, 2, 3, 4]
    P = Propagator(g)
    P.set_survey(shots, stf)
    P.set_model(*[torch.from_numpy(m) for m in true])
    obs = P.forward(ids)
    P.set_model(*[torch.from_numpy(m) for m in init])
    out = {}
    for L in (1, 2, 3):
        P.set_lanes(L)
        scratch = [torch.zeros_like(obs) for _ in range(3)]
        P.set_scratch(*scratch)
        P.profile(1)
        P.profile_read()
        J, gl, gm, gr, res = P.gradient(ids, obs, want_residual=True)
        prof = P.profile_read()
        P.profile(0)
        P.set_scratch()
        Jm = P.misfit(ids, obs)
        out[L] = (J, Jm, gl.cpu(), gm.cpu(), gr.cpu(), res.cpu(), [s.cpu() for s in scratch], prof)
    J1, Jm1, gl1, gm1, gr1, res1, scr1, prof1 = out[1]
    assert J1 > 0 and Jm1 == J1
    for L in (2, 3):
        J, Jm, gl, gm, gr, res, scr, prof = out[L]
        assert J == J1 and Jm == J1
        assert torch.equal(res, res1)
        for a, b in zip(scr, scr1):
            assert torch.equal(a, b)
        for a, b in zip((gl, gm, gr), (gl1, gm1, gr1)):
            assert float((a - b).norm() / b.norm()) < 1e-6
        for k in ("stress_fwd", "velocity_fwd", "rev_velocity", "rev_stress", "misfit"):
            assert prof[k]["launches"] == prof1[k]["launches"], k
            assert 0 < prof[k]["timed"] <= prof1[k]["timed"], k  # lane 0 alone is timed
    P.close()


def test_lane_count_is_checked():
    from efwi.engine import Propagator
    from efwi import EfwiError
    g, *_ = _problem()
    P = Propagator(g)
    for bad in (0, 9):
        with pytest.raises(EfwiError):
            P.set_lanes(bad)
    P.set_lanes(8)
    P.set_lanes(1)
    P.close()


def test_graph_replay_matches_eager_launches():
    """Time loops replayed from CUDA graphs (the default) give the eager
    launches' misfit, images and residuals bit for bit, on the first call
    (capture) and on later calls and shots (replay), with one and two
    lanes."""
    from efwi import synthetic
    from efwi.engine import Propagator
    p = synthetic.small(nz=22, nx=24, ny=20, npml=5, nt=60, nshot=3, nrec=10, seed=5,
                        contrast=0.08)
    P = Propagator(p.grid)
    P.set_survey(p.shots, p.stf)
    P.set_model(*[torch.from_numpy(x) for x in p.params("true")])
    P.set_graphs(False)
    obs = P.forward([0, 1, 2])
    P.set_graphs(True)
    assert torch.equal(P.forward([0, 1, 2]), obs)
    assert torch.equal(P.forward([0, 1, 2]), obs)
    P.set_model(*[torch.from_numpy(x) for x in p.params("init")])
    for lanes in (1, 2):
        P.set_lanes(lanes)
        P.set_graphs(False)
        ref = P.gradient([0, 1, 2], obs, want_residual=True)
        P.set_graphs(True)
        for _ in range(2):
            got = P.gradient([0, 1, 2], obs, want_residual=True)
            assert got[0] == ref[0]
            for x, y in zip(got[1:], ref[1:]):
                assert torch.equal(x, y)


def test_exact_mode_lanes_match_one_lane():
    """Exact gradients on 1, 2 and 3 lanes, each lane with an equal share of
    the checkpoint budget: the same misfit bits and residuals, images equal
    up to the order of the per-shot sums (1e-6 rel-L2), and the source-time
    function gradients of every shot bit for bit."""
    from efwi.engine import Propagator
    g, shots, stf, true, init = _problem()
    ids = [0, 1, 2, 3, 4]
    P = Propagator(g)
    P.set_survey(shots, stf)
    P.set_model(*[torch.from_numpy(m) for m in true])
    obs = P.forward(ids)
    P.set_model(*[torch.from_numpy(m) for m in init])
    P.set_checkpoint_budget(24 * P.state_bytes())
    out = {}
    for L in (1, 2, 3):
        P.set_lanes(L)
        J, gl, gm, gr, gs = P.stf_gradient(ids, obs)
        res = P.gradient(ids, obs, mode="exact", want_residual=True)[4]
        out[L] = (J, [x.cpu() for x in (gl, gm, gr)], gs.cpu(), res.cpu())
    J1, g1, s1, r1 = out[1]
    for L in (2, 3):
        J, gg, ss, rr = out[L]
        assert J == J1
        assert torch.equal(rr, r1)
        assert torch.equal(ss, s1)
        for a, b in zip(gg, g1):
            d = float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
            assert d < 1e-6
