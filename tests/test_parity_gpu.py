"""CUDA engine against the reference's kernels (golden vectors, FP32) and the
FP64 oracle.  Tolerances (rel-L2):

* traces vs the reference's FP32 kernels: 1e-5
* traces, misfit and gradients vs the FP64 oracle: 1e-4
* adjoint source (obs - syn, a small difference of FP32 traces): 3e-4
* batching and launch shapes: bitwise identical
"""
import numpy as np
import pytest
import torch

import oracle
from helpers import case_of, fixture_case, fixture_engine, golden, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _ready():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    oracle.build()


def _prop(prefix, **opts):
    from efwi.engine import Propagator
    g, shots, stf, lam, mu, rho = fixture_engine(prefix)
    P = Propagator(g, **opts)
    P.set_model(torch.from_numpy(lam), torch.from_numpy(mu), torch.from_numpy(rho))
    P.set_survey(shots, stf)
    return P


def test_forward_traces_match_reference_and_oracle():
    d = golden()
    P = _prop("A_")
    tr = P.forward([0, 1]).cpu().numpy()
    assert rel_l2(tr, d["A_traces"]) < 1e-5
    port = np.concatenate([t.ravel() for t in oracle.port().forward(fixture_case("A_"))])
    assert rel_l2(tr, port) < 1e-4


@pytest.mark.parametrize("bx,zchunk,batch", [(4, 16, 1), (8, 7, 2), (4, 5, 2), (8, 64, 1)])
def test_launch_shape_and_batching_are_bitwise_identical(bx, zchunk, batch):
    base = _prop("A_", tile_bx=4, zchunk=16, max_batch=1).forward([0, 1]).cpu()
    other = _prop("A_", tile_bx=bx, zchunk=zchunk, max_batch=batch).forward([0, 1]).cpu()
    assert torch.equal(base, other)


def test_shot_order_and_subsets():
    P = _prop("A_", max_batch=2)
    both = P.forward([0, 1]).cpu()
    rev = P.forward([1, 0]).cpu()
    n0 = both.numel() // 2
    assert torch.equal(both[:n0], rev[n0:]) and torch.equal(both[n0:], rev[:n0])
    assert torch.equal(P.forward([1]).cpu(), both[n0:])


@pytest.mark.parametrize("prefix,if_win", [("B_", False), ("C_", True)])
def test_reference_gradient(prefix, if_win):
    d = golden()
    P = _prop(prefix, if_win=if_win)
    obs = torch.from_numpy(d[prefix + "obs"])
    J, gl, gm, gr, res = P.gradient([0], obs, want_residual=True)
    case = fixture_case(prefix)
    nt, nr = case.nt, case.nrec(0)
    Jp, pl, pm, pr, pres = oracle.port().gradient(
        case, [d[prefix + "obs"].reshape(3, nr, nt).astype(np.float64)], mode=0, if_win=if_win)
    # FP64 oracle: 1e-4
    assert abs(J - Jp) / Jp < 1e-4
    assert rel_l2(gl.cpu(), pl) < 1e-4
    assert rel_l2(gm.cpu(), pm) < 1e-4
    assert rel_l2(gr.cpu(), pr) < 1e-4
    assert rel_l2(res.cpu(), pres[0]) < 3e-4
    # the reference's own FP32 kernels (golden)
    assert abs(J - d[prefix + "misfit"][0]) / d[prefix + "misfit"][0] < 1e-4
    assert rel_l2(gl.cpu(), d[prefix + "glam"]) < 1e-4
    assert rel_l2(gm.cpu(), d[prefix + "gmu"]) < 1e-4
    assert rel_l2(gr.cpu(), d[prefix + "grho"]) < 1e-4


def test_misfit_only_call_matches_gradient_call():
    d = golden()
    P = _prop("B_")
    obs = torch.from_numpy(d["B_obs"])
    J1 = P.misfit([0], obs)
    J2 = P.gradient([0], obs)[0]
    assert J1 == J2


def test_gradient_is_deterministic():
    d = golden()
    P = _prop("B_")
    obs = torch.from_numpy(d["B_obs"])
    a = P.gradient([0], obs)
    b = P.gradient([0], obs)
    for x, y in zip(a[1:], b[1:]):
        assert torch.equal(x, y)


def test_multi_shot_gradient_accumulates_in_shot_order():
    from efwi import synthetic
    from efwi.engine import Propagator
    p = synthetic.small(nz=22, nx=24, ny=20, npml=5, nt=90, nshot=3, nrec=10, seed=9,
                        contrast=0.08)
    lam, mu, rho = p.params("init")
    lt, mt, rt = p.params("true")
    P = Propagator(p.grid, max_batch=3)
    P.set_survey(p.shots, p.stf)
    P.set_model(torch.from_numpy(lt), torch.from_numpy(mt), torch.from_numpy(rt))
    obs = P.forward([0, 1, 2])
    P.set_model(torch.from_numpy(lam), torch.from_numpy(mu), torch.from_numpy(rho))
    J, gl, gm, gr = P.gradient([0, 1, 2], obs)
    oobs = [o.numpy().astype(np.float64) for o in P.split(obs.cpu(), [0, 1, 2])]
    Jp, pl, pm, pr, _ = oracle.port().gradient(case_of(p), oobs, mode=0)
    assert abs(J - Jp) / Jp < 1e-4
    for a, b in ((gl, pl), (gm, pm), (gr, pr)):
        assert rel_l2(a.cpu(), b) < 1e-4


def test_config1_reduced_time_axis_against_oracle():
    """Config-1 grid (84^3 padded, 1024 receivers) with nt = 300: traces and
    reference gradients against the FP64 oracle.  The observed data are half
    the true-model traces, so that the residual is not a small difference of
    nearly equal FP32 traces (whose rounding would dominate it)."""
    from efwi import synthetic
    from efwi.engine import Propagator
    p = synthetic.config1(nt=300)
    lam, mu, rho = p.params("init")
    lt, mt, rt = p.params("true")
    P = Propagator(p.grid)
    P.set_survey(p.shots, p.stf)
    P.set_model(torch.from_numpy(lt), torch.from_numpy(mt), torch.from_numpy(rt))
    tr = P.forward([0])
    port_tr = oracle.port().forward(case_of(p, "true"))
    assert rel_l2(tr.cpu(), port_tr[0]) < 1e-4
    obs = 0.5 * tr
    P.set_model(torch.from_numpy(lam), torch.from_numpy(mu), torch.from_numpy(rho))
    J, gl, gm, gr = P.gradient([0], obs)
    Jp, pl, pm, pr, _ = oracle.port().gradient(
        case_of(p), [obs.cpu().numpy().reshape(3, -1, p.grid.nt).astype(np.float64)], mode=0)
    assert abs(J - Jp) / Jp < 1e-4
    for a, b in ((gl, pl), (gm, pm), (gr, pr)):
        assert rel_l2(a.cpu(), b) < 1e-4


def test_cfl_violation_raises():
    from efwi import CourantError
    from efwi.engine import Propagator
    g, shots, stf, lam, mu, rho = fixture_engine("B_")
    P = Propagator(g)
    with pytest.raises(CourantError, match="Courant"):
        P.set_model(torch.from_numpy(lam) * 1e4, torch.from_numpy(mu) * 1e4, torch.from_numpy(rho))


def test_bad_shot_id_and_call_order_raise():
    from efwi import EfwiError
    from efwi.engine import Propagator
    g, shots, stf, lam, mu, rho = fixture_engine("B_")
    P = Propagator(g)
    with pytest.raises(EfwiError, match="set_model"):
        P.forward([0])
    P.set_model(torch.from_numpy(lam), torch.from_numpy(mu), torch.from_numpy(rho))
    P.set_survey(shots, stf)
    with pytest.raises(EfwiError, match="out of range"):
        P.forward([3])


@pytest.mark.parametrize("bx,zchunk", [(4, 16), (8, 5), (8, 64)])
def test_tma_variant_matches_l1_variant(bx, zchunk):
    """Stencil planes staged by bulk tensor copies against the L1-served
    kernels: forward traces and the misfit are bitwise identical; the fused
    reverse kernels contract a few multiply-adds differently, so their
    gradients agree to 1e-6 (rel-L2)."""
    d = golden()
    a = _prop("A_", tile_bx=bx, zchunk=zchunk, max_batch=2)
    b = _prop("A_", tile_bx=bx, zchunk=zchunk, max_batch=2)
    a.set_variant(0)
    b.set_variant(1)
    assert torch.equal(a.forward([0, 1]).cpu(), b.forward([0, 1]).cpu())
    a = _prop("B_", tile_bx=bx, zchunk=zchunk)
    b = _prop("B_", tile_bx=bx, zchunk=zchunk)
    a.set_variant(0)
    b.set_variant(1)
    obs = torch.from_numpy(d["B_obs"])
    ra, rb = a.gradient([0], obs), b.gradient([0], obs)
    assert ra[0] == rb[0]
    for x, y in zip(ra[1:], rb[1:]):
        assert rel_l2(y.cpu(), x.cpu()) < 1e-6


def test_all_launch_configurations_give_identical_results():
    """The autotuner's knobs (tile, ring depth, occupancy target, z planes
    per CTA) change speed only."""
    d = golden()
    obs = torch.from_numpy(d["B_obs"])
    base = _prop("B_")
    base.set_tuning(0, 8, 0, 8)
    ref_tr = base.forward([0]).cpu()
    ref_g = base.gradient([0], obs)
    for fc, zf, rc, zr in [(1, 4, 1, 4), (2, 12, 2, 16), (3, 5, 3, 3), (0, 64, 1, 64),
                           (1, 2, 4, 2), (2, 3, 5, 6), (1, 4, 6, 4), (0, 8, 7, 3)]:
        P = _prop("B_")
        P.set_tuning(fc, zf, rc, zr)
        assert torch.equal(P.forward([0]).cpu(), ref_tr)
        g = P.gradient([0], obs)
        assert g[0] == ref_g[0]
        for x, y in zip(g[1:], ref_g[1:]):
            assert torch.equal(x, y)


def test_autotuner_keeps_results_and_picks_a_configuration():
    from efwi.autotune import autotune
    d = golden()
    obs = torch.from_numpy(d["B_obs"])
    P = _prop("B_")
    before = P.gradient([0], obs)
    choice = autotune(P, 0, obs, nt_probe=8, zchunks=(4, 8),
                      pair_ids=[0, 0], pair_obs=torch.cat([obs, obs]), lanes_nt=8)
    assert {"fwd_cfg", "rev_cfg", "zchunk_fwd", "zchunk_rev"} <= set(choice)
    assert len(choice["lanes_probe_ms"]) >= 1
    after = P.gradient([0], obs)
    for x, y in zip(before[1:], after[1:]):
        assert torch.equal(x, y)
