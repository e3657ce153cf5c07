"""Learned-preconditioner pipeline on small problems: pseudo-Hessian pairs,
vp gradients through the padding chain, and L-BFGS with and without the
learned step."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _ready():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _obj(mode="exact", seed=5):
    from efwi.preconditioner import VpObjective, layered_problem
    prob = layered_problem(n=24, npml=6, nt=220, shots_side=2, seed=seed, smooth_sigma=4.0)
    return VpObjective(prob, mode=mode)


def test_vp_gradient_finite_differences():
    """Exact vp gradient (chain through replicate padding and lambda(vp))
    against central differences of the misfit, h = 1e-2 relative (the
    misfit difference of two FP32 simulations at h = 1e-3 carries a few %
    of rounding on this small problem), 3 smooth perturbations: 1e-2."""
    from efwi import synthetic
    obj = _obj()
    vp = torch.from_numpy(obj.prob.vp_init).cuda()
    J, g = obj.value_and_grad(vp)
    n = vp.shape[0]
    for k, c in enumerate([(8, 12, 12), (14, 9, 15), (11, 15, 8)]):
        dm = torch.from_numpy(synthetic.gaussian_blob((n, n, n), c, 2.5)).float().cuda() * vp
        h = 1e-2
        fd = (obj.value(vp + h * dm) - obj.value(vp - h * dm)) / (2 * h)
        an = float(torch.sum(g.double() * dm.double()))
        assert abs(fd - an) / abs(fd) < 1e-2, (k, fd, an)


def test_pairs_are_finite_and_normalised():
    from efwi.preconditioner import make_pairs
    pairs = make_pairs(n_pairs=2, n=20, nt=180, nprobe=2)
    for p in pairs:
        assert p["x"].shape == (3, 20, 20, 20) and p["y"].shape == (20, 20, 20)
        assert torch.isfinite(p["x"]).all() and torch.isfinite(p["y"]).all()
        assert abs(float(p["y"].abs().max()) - 1.0) < 1e-5


def test_probe_diagonal_is_positive_and_correlates_with_illumination():
    obj = _obj()
    vp = torch.from_numpy(obj.prob.vp_init).cuda()
    d = obj.probe_diagonal(vp, nprobe=3)
    il = obj.illumination(vp)
    assert float(d.min()) >= 0 and float(il.min()) >= 0
    a = torch.log(d + 1e-12 * d.max()).flatten()
    b = torch.log(il + 1e-12 * il.max()).flatten()
    a, b = a - a.mean(), b - b.mean()
    assert float(torch.sum(a * b) / torch.sqrt(torch.sum(a * a) * torch.sum(b * b))) > 0.5


@pytest.mark.parametrize("mode", ["reference", "exact"])
def test_lbfgs_decreases_misfit_with_and_without_learned_step(mode):
    from efwi.cnn import Preconditioner
    from efwi.preconditioner import lbfgs
    obj = _obj(mode=mode)
    vp0 = torch.from_numpy(obj.prob.vp_init).cuda()
    plain = lbfgs(obj, vp0, iters=3)
    assert plain.misfit[-1] < plain.misfit[0]
    net = Preconditioner(cin=3, seed=1).cuda()
    learned = lbfgs(obj, vp0, iters=3, net=net)
    assert learned.misfit[-1] < learned.misfit[0]
    assert len(learned.seconds) == len(learned.misfit)
