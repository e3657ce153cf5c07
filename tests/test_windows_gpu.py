"""Shot windows (efwi_forward_windows), in one persistent multi-domain
launch of the L1-served stencils or as per-window TMA launches on several
streams, against each window run alone through the single-domain path (L1
kernels): bitwise identical traces, with and without the CUDA graph;
receivers outside their window record zeros."""
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
    nz, nx, ny, np_, nt = 22, 44, 40, 5, 120
    g = Grid(nz, nx, ny, np_, nt, 10.0, 10.0, 10.0, 1e-3, 12.0)
    rng = np.random.default_rng(3)
    mz, mx, my = nz - 2 * np_, nx - 2 * np_, ny - 2 * np_
    vp = (2200.0 + 300.0 * rng.random((mz, mx, my))).astype(np.float32)
    vs = (vp / 1.732).astype(np.float32)
    rho = (310.0 * vp ** 0.25).astype(np.float32)
    lam, mu, rh = synthetic.elastic_params(vp, vs, rho, np_)
    xs = np.arange(np_, nx - np_, 3)
    ys = np.arange(np_, ny - np_, 3)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    zr = np.full(X.size, np_ + 1, np.int32)
    shots = [Shot(src=(np_ + 2, 14, 12), z_rec=zr, x_rec=X.ravel().astype(np.int32),
                  y_rec=Y.ravel().astype(np.int32)),
             Shot(src=(np_ + 3, 28, 25), z_rec=zr, x_rec=X.ravel().astype(np.int32),
                  y_rec=Y.ravel().astype(np.int32)),
             Shot(src=(np_ + 2, 22, 20), z_rec=zr, x_rec=X.ravel().astype(np.int32),
                  y_rec=Y.ravel().astype(np.int32))]
    stf = np.stack([synthetic.ricker(12.0 + k, nt, 1e-3) for k in range(3)])
    windows = [(2, 0, 27, 26), (12, 10, 32, 30), (0, 0, 44, 40)]
    return g, shots, stf, (lam, mu, rh), windows


def _alone(g, shot, stf_row, model, w, bx, zchunk):
    """The shot on its window as its own grid (single-domain L1 path)."""
    from efwi.engine import Grid, Propagator, Shot
    x0, y0, nxw, nyw = w
    gw = Grid(g.nz, nxw, nyw, g.npml, g.nt, g.dz, g.dx, g.dy, g.dt, g.f0)
    inside = ((shot.x_rec >= x0) & (shot.x_rec < x0 + nxw) & (shot.y_rec >= y0) &
              (shot.y_rec < y0 + nyw))
    sw = Shot(src=(shot.src[0], shot.src[1] - x0, shot.src[2] - y0), z_rec=shot.z_rec[inside],
              x_rec=(shot.x_rec[inside] - x0).astype(np.int32),
              y_rec=(shot.y_rec[inside] - y0).astype(np.int32))
    P = Propagator(gw, tile_bx=bx, zchunk=zchunk)
    P.set_variant(0)
    P.set_survey([sw], stf_row[None, :])
    P.set_model(*[torch.from_numpy(np.ascontiguousarray(m[:, x0:x0 + nxw, y0:y0 + nyw]))
                  for m in model])
    tr = P.forward([0]).view(3, int(inside.sum()), g.nt).cpu()
    P.close()
    return inside, tr


@pytest.mark.parametrize("bx,zchunk", [(4, 8), (8, 5)])
@pytest.mark.parametrize("graph", [False, True])
def test_windows_match_single_domain_runs(bx, zchunk, graph):
    from efwi.engine import Propagator
    g, shots, stf, model, windows = _problem()
    P = Propagator(g, tile_bx=bx, zchunk=zchunk)
    P.set_variant(0)
    P.set_survey(shots, stf)
    P.set_model(*[torch.from_numpy(m) for m in model])
    out = P.forward_windows([0, 1, 2], windows, use_graph=graph).cpu()
    parts = P.split(out, [0, 1, 2])
    for k in range(3):
        inside, tr = _alone(g, shots[k], stf[k], model, windows[k], bx, zchunk)
        assert torch.equal(parts[k][:, torch.from_numpy(inside), :], tr)
        assert float(parts[k][:, torch.from_numpy(~inside), :].abs().max() if (~inside).any() else 0) == 0.0


def test_full_grid_window_equals_plain_forward():
    from efwi.engine import Propagator
    g, shots, stf, model, _ = _problem()
    P = Propagator(g, tile_bx=4, zchunk=8)
    P.set_variant(0)
    P.set_survey(shots, stf)
    P.set_model(*[torch.from_numpy(m) for m in model])
    full = [(0, 0, g.nx, g.ny)] * 3
    assert torch.equal(P.forward_windows([0, 1, 2], full).cpu(), P.forward([0, 1, 2]).cpu())


@pytest.mark.parametrize("cfg,zchunk", [(0, 8), (1, 5), (3, 3)])
def test_tma_windows_match_single_domain_runs(cfg, zchunk):
    from efwi.engine import Propagator
    g, shots, stf, model, windows = _problem()
    P = Propagator(g, zchunk=zchunk)
    P.set_variant(1)
    P.set_tuning(cfg, zchunk, 0, 0)
    P.set_survey(shots, stf)
    P.set_model(*[torch.from_numpy(m) for m in model])
    out = P.forward_windows([0, 1, 2], windows).cpu()
    parts = P.split(out, [0, 1, 2])
    for k in range(3):
        inside, tr = _alone(g, shots[k], stf[k], model, windows[k], 4, zchunk)
        assert torch.equal(parts[k][:, torch.from_numpy(inside), :], tr)
        assert float(parts[k][:, torch.from_numpy(~inside), :].abs().max() if (~inside).any() else 0) == 0.0


def test_tma_windows_on_eight_streams_equal_the_multi_domain_launch():
    """11 windows (more than the 8 stream groups; shots repeated on other
    windows): the per-window TMA launches give the multi-domain launch's
    bits, receivers of every group included."""
    from efwi.engine import Propagator
    g, shots, stf, model, _ = _problem()
    ids = [0, 0, 0, 1, 1, 1, 2, 2, 2, 0, 1]
    wins = [(2, 0, 27, 26), (0, 0, 30, 30), (5, 3, 20, 20), (12, 10, 32, 30), (18, 15, 20, 20),
            (10, 8, 34, 32), (0, 0, 44, 40), (10, 10, 25, 22), (15, 12, 16, 17), (3, 2, 24, 28),
            (20, 20, 24, 20)]
    P = Propagator(g, tile_bx=4, zchunk=4)
    P.set_survey(shots, stf)
    P.set_model(*[torch.from_numpy(m) for m in model])
    P.set_variant(0)
    ref = P.forward_windows(ids, wins, use_graph=True).cpu()
    P.set_variant(1)
    out = P.forward_windows(ids, wins).cpu()
    assert float(ref.abs().max()) > 0
    assert torch.equal(out, ref)


@pytest.mark.parametrize("mode", ["reference", "exact"])
def test_window_gradients_match_each_window_alone(mode):
    """efwi_gradient_windows against each window's problem run alone (its
    own grid, the window of the model, the receivers inside it): the misfit
    is the sum of the windows' misfits and the images are the windows'
    images added at their places, bit for bit."""
    from efwi.engine import Grid, Propagator, Shot
    g, shots, stf, model, windows = _problem()
    ids = [0, 1, 2]
    true = [m * np.float32(1.03) for m in model]
    P = Propagator(g)
    P.set_survey(shots, stf)
    P.set_model(*[torch.from_numpy(m) for m in true])
    obs = P.forward(ids)
    P.set_model(*[torch.from_numpy(m) for m in model])
    J, gl, gm, gr = P.gradient_windows(ids, windows, obs, mode=mode)
    parts = P.split(obs, ids)
    Jsum = 0.0
    acc = [np.zeros(g.shape, np.float32) for _ in range(3)]
    for k, (shot, w) in enumerate(zip(shots, windows)):
        x0, y0, nxw, nyw = w
        gw = Grid(g.nz, nxw, nyw, g.npml, g.nt, g.dz, g.dx, g.dy, g.dt, g.f0)
        inside = ((shot.x_rec >= x0) & (shot.x_rec < x0 + nxw) & (shot.y_rec >= y0) &
                  (shot.y_rec < y0 + nyw))
        sw = Shot(src=(shot.src[0], shot.src[1] - x0, shot.src[2] - y0),
                  z_rec=shot.z_rec[inside], x_rec=(shot.x_rec[inside] - x0).astype(np.int32),
                  y_rec=(shot.y_rec[inside] - y0).astype(np.int32))
        Q = Propagator(gw)
        Q.set_lanes(1)
        Q.set_survey([sw], stf[k][None, :])
        Q.set_model(*[torch.from_numpy(np.ascontiguousarray(m[:, x0:x0 + nxw, y0:y0 + nyw]))
                      for m in model])
        ob = parts[k].view(3, shot.nrec, g.nt)[:, torch.from_numpy(inside).to(obs.device)]
        Jk, *gk = Q.gradient([0], ob.contiguous().reshape(-1), mode=mode)
        Jsum += Jk
        for a, b in zip(acc, gk):
            a[:, x0:x0 + nxw, y0:y0 + nyw] += b.cpu().numpy()
        Q.close()
    assert J == Jsum
    for a, b in zip((gl, gm, gr), acc):
        assert np.array_equal(a.cpu().numpy(), b)
