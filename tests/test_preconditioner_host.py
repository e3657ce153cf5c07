"""Host side of the preconditioner pipeline: seeded problems (no GPU)."""
import numpy as np


def test_layered_problem_is_seeded_and_stable():
    from efwi.preconditioner import layered_problem
    a = layered_problem(n=24, npml=6, nt=200, seed=3)
    b = layered_problem(n=24, npml=6, nt=200, seed=3)
    c = layered_problem(n=24, npml=6, nt=200, seed=4)
    assert np.array_equal(a.vp_true, b.vp_true) and not np.array_equal(a.vp_true, c.vp_true)
    assert 1600 < a.vp_true.min() and a.vp_true.max() < 4500
    g = a.grid
    courant = a.vp_true.max() * g.dt * np.sqrt(2) * (9 / 8 + 1 / 24) / g.dx
    assert courant < 1.0
    assert len(a.shots) == 4 and all(0 <= s.src[0] < g.nz for s in a.shots)
    n = 24
    for s in a.shots:
        assert s.x_rec.max() < g.nx - g.npml and s.y_rec.max() < g.ny - g.npml


class _Quadratic:
    """vp objective 0.5 sum h (v - v*)^2 on the CPU, h falling by three
    orders of magnitude with depth (like the illumination of a surface
    survey); the illumination is h itself."""

    def __init__(self, n: int = 12, seed: int = 0):
        import torch
        gen = torch.Generator().manual_seed(seed)
        z = torch.arange(n, dtype=torch.float64)
        self.h = (10.0 ** (-3.0 * z / (n - 1)))[:, None, None] * \
            (1.0 + 0.5 * torch.rand(n, n, n, generator=gen, dtype=torch.float64))
        self.vp_true = 2500.0 + 200.0 * torch.rand(n, n, n, generator=gen, dtype=torch.float64)
        self.dev = torch.device("cpu")
        self.evals = 0

    def value(self, v):
        self.evals += 1
        return float(0.5 * (self.h * (v - self.vp_true) ** 2).sum())

    def value_and_grad(self, v):
        return self.value(v), self.h * (v - self.vp_true)

    def illumination(self, v):
        return self.h.clone()


def _ideal_net(x):
    """The map the CNN is trained towards on this objective: the gradient
    divided by the illumination, normalised (inverted from the features)."""
    illum = 10.0 ** ((x[2] - 1.0) * 6.0) - 1e-6
    d = x[0] / illum
    return d / d.abs().max()


def test_learned_h0_preconditions_the_quasi_newton_step():
    import torch
    from efwi.preconditioner import lbfgs
    obj = _Quadratic()
    v0 = torch.full_like(obj.vp_true, 2500.0)
    plain = lbfgs(obj, v0, iters=8)
    learned = lbfgs(_Quadratic(), v0, iters=8, net=_ideal_net, net_mode="h0")
    # the ideal map is the exact inverse Hessian up to a scalar: the second
    # iteration lands on the minimum, where plain L-BFGS has barely started
    assert learned.learned_accepted >= 2
    assert learned.misfit[2] < 1e-12 * learned.misfit[0]
    assert plain.misfit[-1] > 1e-3 * plain.misfit[0]
    assert learned.model_rel_l2[-1] < 1e-6 < plain.model_rel_l2[-1]


def test_learned_h0_falls_back_to_the_plain_step():
    """A map that points uphill is never used: the run is the plain one."""
    import torch
    from efwi.preconditioner import lbfgs
    v0 = torch.full((12, 12, 12), 2500.0, dtype=torch.float64)
    plain = lbfgs(_Quadratic(), v0, iters=6)
    bad = lbfgs(_Quadratic(), v0, iters=6, net=lambda x: -x[0], net_mode="h0")
    assert bad.learned_accepted == 0
    assert bad.misfit == plain.misfit


def test_net_mode_is_checked():
    import pytest
    import torch
    from efwi.preconditioner import lbfgs
    with pytest.raises(ValueError):
        lbfgs(_Quadratic(), torch.full((12, 12, 12), 2500.0, dtype=torch.float64), iters=1,
              net_mode="other")


class _TinyQuadratic(_Quadratic):
    """The same objective in FP32 with the misfit scaled by 1e-27, so that
    squares of the gradient entries underflow FP32: the L-BFGS recursion
    must not depend on the scale of the misfit."""

    SCALE = 1e-27

    def __init__(self):
        super().__init__()
        self.h = (self.h * self.SCALE).float()
        self.vp_true = self.vp_true.float()


def test_lbfgs_steps_on_gradients_whose_squares_underflow_fp32():
    import torch
    from efwi.preconditioner import lbfgs
    obj = _TinyQuadratic()
    g0 = obj.value_and_grad(torch.full_like(obj.vp_true, 2500.0))[1]
    assert float(torch.sum(g0 * g0)) == 0.0  # the FP32 inner product underflows
    res = lbfgs(obj, torch.full_like(obj.vp_true, 2500.0), iters=6)
    assert len(res.misfit) == 7
    assert res.misfit[-1] < 0.5 * res.misfit[0]


def test_training_loss_sees_direction_only():
    import torch
    from efwi.preconditioner import _cosine_loss
    g = torch.Generator().manual_seed(1)
    a = torch.randn(3, 4, 5, generator=g, dtype=torch.float64)
    assert abs(float(_cosine_loss(3.0 * a, a))) < 1e-12
    assert abs(float(_cosine_loss(-a, a)) - 2.0) < 1e-12
    p = torch.randn(3, 4, 5, generator=g, dtype=torch.float64, requires_grad=True)
    _cosine_loss(p, a).backward()
    # the loss does not change along p itself: its gradient is orthogonal to p
    assert abs(float(torch.sum(p.grad * p.detach()))) < 1e-10
