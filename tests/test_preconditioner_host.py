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
