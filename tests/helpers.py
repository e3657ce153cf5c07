"""Test helpers: conversions between engine problems and oracle cases."""
import numpy as np

import oracle
from efwi.synthetic import Problem


def case_of(p: Problem, which: str = "init", dtype=np.float64, if_win=False) -> "oracle.Case":
    lam, mu, rho = p.params(which)
    g = p.grid
    win = None
    if if_win:
        win = [(s.win_start, s.win_end, s.weights, s.src_weight) for s in p.shots]
    return oracle.Case(g.nz, g.nx, g.ny, g.npml, g.nt, float(np.float32(g.dz)),
                       float(np.float32(g.dx)), float(np.float32(g.dy)),
                       float(np.float32(g.dt)), g.f0,
                       lam.astype(dtype), mu.astype(dtype), rho.astype(dtype),
                       [tuple(s.src) for s in p.shots],
                       [(s.z_rec, s.x_rec, s.y_rec) for s in p.shots],
                       p.stf.astype(dtype), win)


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d > 0 else 1.0))


GOLDEN = None


def golden():
    global GOLDEN
    if GOLDEN is None:
        import os
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_small.npz")
        GOLDEN = dict(np.load(path))
    return GOLDEN


def fixture_case(prefix: str, which: str = "init", dtype=np.float64) -> "oracle.Case":
    """Oracle case of a golden fixture (inputs as stored)."""
    d = golden()
    gi, gf = d[prefix + "grid_i"], d[prefix + "grid_f"]
    sfx = "" if which == "init" else "_true"
    win = None
    if prefix + "win" in d:
        w, sw = d[prefix + "win"], d[prefix + "src_weight"]
        win = [(w[k, 0], w[k, 1], w[k, 2], float(sw[k])) for k in range(len(sw))]
    return oracle.Case(int(gi[0]), int(gi[1]), int(gi[2]), int(gi[3]), int(gi[4]),
                       float(gf[0]), float(gf[1]), float(gf[2]), float(gf[3]), float(gf[4]),
                       d[prefix + "lam" + sfx].astype(dtype), d[prefix + "mu" + sfx].astype(dtype),
                       d[prefix + "rho" + sfx].astype(dtype),
                       [tuple(int(v) for v in s) for s in d[prefix + "src"]],
                       [(r[0], r[1], r[2]) for r in d[prefix + "rec"]],
                       d[prefix + "stf"].astype(dtype), win)


def fixture_engine(prefix: str):
    """(Grid, [Shot], stf, lam, mu, rho) of a golden fixture for the engine."""
    from efwi.engine import Grid, Shot
    d = golden()
    gi, gf = d[prefix + "grid_i"], d[prefix + "grid_f"]
    g = Grid(int(gi[0]), int(gi[1]), int(gi[2]), int(gi[3]), int(gi[4]), float(gf[0]),
             float(gf[1]), float(gf[2]), float(gf[3]), float(gf[4]))
    shots = []
    for k, (s, r) in enumerate(zip(d[prefix + "src"], d[prefix + "rec"])):
        sh = Shot(src=tuple(int(v) for v in s), z_rec=r[0], x_rec=r[1], y_rec=r[2])
        if prefix + "win" in d:
            w = d[prefix + "win"][k]
            sh.win_start, sh.win_end, sh.weights = w[0], w[1], w[2]
            sh.src_weight = float(d[prefix + "src_weight"][k])
        shots.append(sh)
    return g, shots, d[prefix + "stf"], d[prefix + "lam"], d[prefix + "mu"], d[prefix + "rho"]


# (axis, C-PML slot) of state components 9..26, the oracle's order
PSI_AXIS_SLOT = [(0, 0), (1, 1), (2, 1), (0, 1), (1, 0), (2, 2), (0, 2), (1, 2), (2, 0),
                 (0, 3), (1, 3), (2, 3), (0, 4), (1, 4), (1, 5), (2, 5), (2, 4), (0, 5)]


def step_support(g):
    """Cells the step updates: fields on [2, n-3]^3; memory variables there
    and inside their slab (x/y velocity-stage slabs with quirk Q2)."""
    nz, nx, ny, np_ = g.nz, g.nx, g.ny, g.npml
    z = np.arange(nz)[:, None, None]
    x = np.arange(nx)[None, :, None]
    y = np.arange(ny)[None, None, :]
    inner = (z >= 2) & (z <= nz - 3) & (x >= 2) & (x <= nx - 3) & (y >= 2) & (y <= ny - 3)
    coords = (z, x, y)
    ns = (nz, nx, ny)
    m = np.zeros((27, nz, nx, ny), bool)
    m[:9] = inner
    for k, (ax, slot) in enumerate(PSI_AXIS_SLOT):
        c, n = coords[ax], ns[ax]
        if slot >= 3 and ax > 0:
            slab = (c < np_) | (c > n - np_)
        else:
            slab = (c < np_) | (c > n - np_ - 1)
        m[9 + k] = inner & slab
    return m
