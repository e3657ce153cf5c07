"""Exact discrete adjoint on the GPU (EFWI_MODE_EXACT, efwi_step).

Tolerances, stated per test:
* one forward step and one transposed step vs the FP64 oracle: rel-L2 1e-5
  per state component;
* dot-product test <A x, A x> = <x, A^T A x> in FP32: 1e-5 relative;
* exact gradients and misfit vs the FP64 oracle (mode 1): rel-L2 1e-4;
* central finite differences of the GPU misfit (h = 1e-3 relative, smooth
  perturbations): median 5e-3, worst 5e-2 relative -- the misfit comes
  from FP32 traces, so the difference of two misfits carries their
  rounding (the FP64 oracle passes the same test at 1e-6);
* any checkpoint budget: bitwise identical gradients.
"""
import numpy as np
import pytest
import torch

import oracle
from helpers import PSI_AXIS_SLOT, case_of, rel_l2, step_support as _support

pytestmark = pytest.mark.gpu

@pytest.fixture(scope="module", autouse=True)
def _ready():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    oracle.build()


def _engine(p, which="init", **opts):
    from efwi.engine import Propagator
    P = Propagator(p.grid, **opts)
    P.set_survey(p.shots, p.stf)
    lam, mu, rho = p.params(which)
    P.set_model(torch.from_numpy(lam), torch.from_numpy(mu), torch.from_numpy(rho))
    return P


def _small(seed=1):
    from efwi import synthetic
    return synthetic.small(nz=16, nx=18, ny=20, npml=4, nt=40, nshot=1, nrec=6, seed=seed)


def test_forward_step_matches_oracle():
    p = _small()
    g = p.grid
    P = _engine(p)
    x = np.random.default_rng(0).standard_normal((27, g.nz, g.nx, g.ny)).astype(np.float32)
    ours = P.step(torch.from_numpy(x)).cpu().numpy()
    ref = oracle.port().step(case_of(p), x.astype(np.float64).ravel()).reshape(x.shape)
    for k in range(27):
        assert rel_l2(ours[k], ref[k]) < 1e-5, k


def test_transposed_step_matches_oracle():
    p = _small()
    g = p.grid
    P = _engine(p)
    m = _support(g)
    y = np.random.default_rng(1).standard_normal(m.shape).astype(np.float32) * m
    ours = P.step(torch.from_numpy(y), transpose=True).cpu().numpy() * m
    ref = oracle.port().step_T(case_of(p), y.astype(np.float64).ravel()).reshape(y.shape) * m
    for k in range(27):
        assert rel_l2(ours[k], ref[k]) < 1e-5, k


def test_dot_product_fp32():
    p = _small(seed=2)
    g = p.grid
    P = _engine(p)
    m = _support(g)
    x = torch.from_numpy(np.random.default_rng(3).standard_normal(m.shape).astype(np.float32) * m)
    ax = P.step(x)
    atax = P.step(ax, transpose=True)
    lhs = torch.sum(ax.double() * ax.double()).item()
    rhs = torch.sum(x.double().to(atax.device) * atax.double()).item()
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


def _problem(nshot=1, seed=4):
    from efwi import synthetic
    return synthetic.small(nz=18, nx=20, ny=22, npml=5, nt=70, nshot=nshot, nrec=8, seed=seed,
                           contrast=0.08)


def _obs(p):
    Pt = _engine(p, "true")
    return Pt.forward(list(range(len(p.shots))))


@pytest.mark.parametrize("nshot", [1, 2])
def test_exact_gradient_matches_oracle(nshot):
    p = _problem(nshot)
    obs = _obs(p)
    P = _engine(p)
    ids = list(range(nshot))
    J, gl, gm, gr, res = P.gradient(ids, obs, mode="exact", want_residual=True)
    oobs = [o.numpy().astype(np.float64) for o in P.split(obs.cpu(), ids)]
    Jp, pl, pm, pr, pres = oracle.port().gradient(case_of(p), oobs, mode=1)
    assert abs(J - Jp) / Jp < 1e-4
    for a, b in ((gl, pl), (gm, pm), (gr, pr)):
        assert rel_l2(a.cpu(), b) < 1e-4
    # the misfit and adjoint source are those of the reference mode
    J0, _, _, _, res0 = P.gradient(ids, obs, mode="reference", want_residual=True)
    assert J == J0 and torch.equal(res, res0)


def test_checkpoint_budget_gives_identical_gradients():
    p = _problem()
    obs = _obs(p)
    P = _engine(p)
    state = P.state_bytes()
    nt = p.grid.nt
    out = {}
    for slots in (nt, 4, 2):
        P.set_checkpoint_budget(slots * state)
        out[slots] = P.gradient([0], obs, mode="exact")
        st = P.checkpoint_stats()
        plan = __import__("efwi")._lib.checkpoint_plan(nt, min(slots, nt - 1))
        assert st["forward_steps"] == plan["forward_steps"]
        assert st["slots"] == plan["slots_used"]
    for slots in (4, 2):
        assert out[slots][0] == out[nt][0]
        for a, b in zip(out[slots][1:], out[nt][1:]):
            assert torch.equal(a, b)


def test_too_small_budget_is_an_error():
    from efwi import EfwiError
    p = _problem()
    P = _engine(p)
    P.set_checkpoint_budget(0)
    with pytest.raises(EfwiError):
        P.gradient([0], _obs(p), mode="exact")


def test_exact_gradient_finite_differences():
    """20 smooth (Gaussian-blob) perturbations of lambda, mu or rho."""
    from efwi import synthetic
    p = _problem()
    obs = _obs(p)
    P = _engine(p)
    J, gl, gm, gr = P.gradient([0], obs, mode="exact")
    grads = {"lam": gl.cpu().numpy(), "mu": gm.cpu().numpy(), "rho": gr.cpu().numpy()}
    lam, mu, rho = p.params("init")
    base = {"lam": lam, "mu": mu, "rho": rho}
    g = p.grid
    rng = np.random.default_rng(11)
    h = 1e-3
    errs = []
    for k in range(20):
        key = ("lam", "mu", "rho")[k % 3]
        c = (rng.uniform(g.npml + 2, g.nz - g.npml - 3), rng.uniform(g.npml + 2, g.nx - g.npml - 3),
             rng.uniform(g.npml + 2, g.ny - g.npml - 3))
        blob = synthetic.gaussian_blob((g.nz, g.nx, g.ny), c, 2.0)
        dm = (base[key] * blob).astype(np.float64)

        def J_at(sign):
            m = dict(base)
            m[key] = (base[key] + sign * h * dm).astype(np.float32)
            P.set_model(torch.from_numpy(m["lam"]), torch.from_numpy(m["mu"]),
                        torch.from_numpy(m["rho"]))
            return P.misfit([0], obs)

        fd = (J_at(1) - J_at(-1)) / (2 * h)
        an = float(np.sum(grads[key].astype(np.float64) * dm))
        errs.append(abs(fd - an) / max(abs(fd), 1e-30))
    assert np.median(errs) < 5e-3 and max(errs) < 5e-2, errs


def test_config3_grid_checkpointed_equals_full_storage():
    """Config-3 grid (96^3 model, 120^3 padded, np 12) with nt = 160: the
    4 GiB budget (49 slots) and storage of every state give bitwise equal
    gradients."""
    from efwi.engine import Grid, Shot
    from efwi import synthetic
    n, np_, nt = 120, 12, 160
    g = Grid(n, n, n, np_, nt, 10.0, 10.0, 10.0, 1e-3, 10.0)
    m = n - 2 * np_
    vp = np.full((m, m, m), 2500.0, np.float32)
    vp[m // 2:] = 3000.0
    vs = (vp / 1.732).astype(np.float32)
    rho = (310.0 * vp ** 0.25).astype(np.float32)
    zr, xr, yr = synthetic._receivers_grid(16, 6, 1, 2, np_)
    shot = Shot(src=(np_ + 5, n // 2, n // 2), z_rec=zr, x_rec=xr, y_rec=yr)
    stf = synthetic.ricker(10.0, nt, 1e-3)[None, :]
    lam, mu, rh = synthetic.elastic_params(vp, vs, rho, np_)
    lam_t, mu_t, rh_t = synthetic.elastic_params(vp * 1.02, vs, rho, np_)
    from efwi.engine import Propagator
    P = Propagator(g)
    P.set_survey([shot], stf)
    P.set_model(torch.from_numpy(lam_t), torch.from_numpy(mu_t), torch.from_numpy(rh_t))
    obs = P.forward([0])
    P.set_model(torch.from_numpy(lam), torch.from_numpy(mu), torch.from_numpy(rh))
    P.set_checkpoint_budget(4 << 30)
    a = P.gradient([0], obs, mode="exact")
    assert P.checkpoint_stats()["slots"] == 49
    P.set_checkpoint_budget(nt * P.state_bytes())
    b = P.gradient([0], obs, mode="exact")
    assert P.checkpoint_stats()["forward_steps"] == nt - 1
    assert a[0] == b[0]
    for x, y in zip(a[1:], b[1:]):
        assert torch.equal(x, y)


def test_autograd_function_chains_through_vp():
    """ElasticMisfit's backward returns the exact images scaled by the
    incoming gradient, and torch's chain rule carries them to vp."""
    from efwi.autograd import misfit
    p = _problem()
    obs = _obs(p)
    P = _engine(p)
    lam, mu, rho = (torch.from_numpy(x).cuda() for x in p.params("init"))
    vp = torch.sqrt((lam + 2 * mu) / rho).requires_grad_(True)
    vs = torch.sqrt(mu / rho)
    lam2 = (vp * vp - 2 * vs * vs) * rho
    mu2 = vs * vs * rho
    P.set_model(lam2.detach(), mu2.detach(), rho)
    J, gl, gm, gr = P.gradient([0], obs, mode="exact")
    loss = 3.0 * misfit(lam2, mu2, rho, P, [0], obs)
    loss.backward()
    assert abs(loss.item() - 3.0 * J) / J < 1e-6
    expect = 3.0 * (gl + 0 * gm) * 2 * vp.detach() * rho
    assert rel_l2(vp.grad.cpu(), expect.cpu()) < 1e-5


def test_exact_tile_width_is_bitwise_neutral():
    p = _problem(nshot=2)
    obs = _obs(p)
    a = _engine(p, tile_bx=4).gradient([0, 1], obs, mode="exact")
    b = _engine(p, tile_bx=8).gradient([0, 1], obs, mode="exact")
    assert a[0] == b[0]
    for x, y in zip(a[1:], b[1:]):
        assert torch.equal(x, y)


def test_adjoint_of_the_residual_is_the_exact_gradient():
    """J^T w with w = dJ/dsyn = -2 res gives the exact gradient: bitwise on
    one lane (the same per-shot sums in the same order); with two shot lanes
    the gradient adds the lanes' images in lane order, 1e-6."""
    p = _problem(nshot=2)
    obs = _obs(p)
    P = _engine(p)
    P.set_lanes(1)
    J, gl, gm, gr, res = P.gradient([0, 1], obs, mode="exact", want_residual=True)
    al, am, ar = P.adjoint([0, 1], -2.0 * res)
    for a, b in ((al, gl), (am, gm), (ar, gr)):
        assert torch.equal(a, b)
    P.set_lanes(2)
    J2, gl2, gm2, gr2 = P.gradient([0, 1], obs, mode="exact")
    assert J2 == J
    for a, b in ((al, gl2), (am, gm2), (ar, gr2)):
        assert rel_l2(a.cpu(), b.cpu()) < 1e-6


def test_illumination_matches_oracle():
    """Diagonal pseudo-Hessian (Shin et al. 2001) vs the FP64 oracle, rel-L2 1e-4."""
    p = _problem(nshot=2)
    P = _engine(p)
    hl, hm, hr = P.illumination([0, 1])
    ol, om, orr = oracle.port().illumination(case_of(p))
    for a, b in ((hl, ol), (hm, om), (hr, orr)):
        assert rel_l2(a.cpu(), b) < 1e-4
    assert float(hl.min()) >= 0 and float(hm.min()) >= 0 and float(hr.min()) >= 0


def test_stf_gradient_matches_central_differences():
    """dJ/dstf of the exact mode: J is quadratic in the source-time function,
    so central differences carry only FP32 rounding; rel 2e-3 on two smooth
    directions of shot 0's (untapered) stf row."""
    p = _problem(nshot=2)
    obs = _obs(p)
    P = _engine(p)
    J, gl, gm, gr, gs = P.stf_gradient([0, 1], obs)
    assert gs.shape == (2, p.grid.nt)
    t = np.arange(p.grid.nt)
    for k, d in enumerate([p.stf[0].astype(np.float64),
                           np.exp(-((t - 30.0) / 6.0) ** 2) * np.abs(p.stf[0]).max()]):
        h = 1e-3

        def J_at(sign):
            stf = p.stf.astype(np.float64).copy()
            stf[0] += sign * h * d
            P.set_survey(p.shots, stf.astype(np.float32))
            return P.misfit([0, 1], obs)

        fd = (J_at(1) - J_at(-1)) / (2 * h)
        an = float(np.sum(gs[0].cpu().numpy().astype(np.float64) * d))
        assert abs(fd - an) / abs(fd) < 2e-3, (k, fd, an)
    P.set_survey(p.shots, p.stf)
    # turning the output off leaves the images unchanged
    J2, a, b, c = P.gradient([0, 1], obs, mode="exact")
    assert J2 == J and torch.equal(a, gl) and torch.equal(b, gm) and torch.equal(c, gr)


@pytest.mark.parametrize("bx,zchunk", [(4, 8), (8, 5), (4, 1), (8, 64)])
def test_staged_adjoint_kernels_match_l1_kernels(bx, zchunk):
    """The exact adjoint kernels with bulk-copy staged planes (TMA variant)
    against the L1 kernels, for both tiles and any z chunk: the same misfit
    (the forward sweep is shared) and gradients to 1e-6 rel-L2 (the two
    compile the same per-cell expressions, but may contract multiply-adds
    differently)."""
    p = _problem(nshot=1, seed=6)
    obs = _obs(p)
    res = []
    for variant in (0, 1):
        P = _engine(p, tile_bx=bx, zchunk=zchunk)
        P.set_tuning(1, zchunk, 4, zchunk)
        P.set_variant(variant)
        res.append(P.gradient([0], obs, mode="exact"))
    assert res[0][0] == res[1][0]
    for x, y in zip(res[0][1:], res[1][1:]):
        d = rel_l2(y.cpu(), x.cpu())
        print(f"TMA vs L1 exact gradient rel-L2 {d:.3e}")
        assert d < 1e-6
