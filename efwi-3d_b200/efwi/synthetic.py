"""Seeded synthetic problems of the benchmark configurations.

The reference publishes no datasets for this operator; these builders make
models, wavelets and acquisition geometries of the stated shapes, sizes and
value ranges.  Units follow the reference's FWI_3d convention: vp, vs in m/s
and rho in kg/m^3 on the model grid; the engine receives
rho' = rho / 1e3, lambda = (vp^2 - 2 vs^2) rho', mu = vs^2 rho' on the
padded grid (replicate padding).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from .engine import Grid, Shot


def ricker(f0: float, nt: int, dt: float) -> np.ndarray:
    """Ricker wavelet delayed by 1.2/f0 (fwi_utils.py:92-96 without the
    running sum)."""
    e = (np.pi * f0) ** 2
    t = np.arange(nt) * dt - 1.2 / f0
    return ((1.0 - 2.0 * e * t * t) * np.exp(-e * t * t)).astype(np.float32)


def pad_edge(v: np.ndarray, npml: int) -> np.ndarray:
    return np.pad(v, npml, mode="edge")


def elastic_params(vp: np.ndarray, vs: np.ndarray, rho_kgm3: np.ndarray, npml: int):
    """Padded lambda, mu, rho' (float32) from model-grid vp, vs, rho."""
    vp_p, vs_p, r_p = (pad_edge(np.asarray(a, np.float32), npml) for a in (vp, vs, rho_kgm3))
    rho = r_p / np.float32(1e3)
    lam = (vp_p ** 2 - np.float32(2.0) * vs_p ** 2) * rho
    mu = vs_p ** 2 * rho
    return lam.astype(np.float32), mu.astype(np.float32), rho.astype(np.float32)


def gaussian_blob(shape, center, sigma) -> np.ndarray:
    z, x, y = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in shape], indexing="ij")
    r2 = (z - center[0]) ** 2 + (x - center[1]) ** 2 + (y - center[2]) ** 2
    return np.exp(-r2 / (2.0 * sigma * sigma))


def smooth(v: np.ndarray, sigma: float) -> np.ndarray:
    from scipy.ndimage import gaussian_filter
    return gaussian_filter(v.astype(np.float64), sigma=sigma, mode="nearest").astype(np.float32)


@dataclass
class Problem:
    name: str
    grid: Grid
    shots: List[Shot]
    stf: np.ndarray          # [nshot, nt]
    vp_true: np.ndarray      # model grid
    vs_true: np.ndarray
    rho_true: np.ndarray     # kg/m^3
    vp_init: np.ndarray
    vs_init: np.ndarray
    rho_init: np.ndarray

    @property
    def npml(self) -> int:
        return self.grid.npml

    def params(self, which: str = "init"):
        if which == "true":
            return elastic_params(self.vp_true, self.vs_true, self.rho_true, self.npml)
        return elastic_params(self.vp_init, self.vs_init, self.rho_init, self.npml)

    @property
    def cell_steps(self) -> int:
        """Cell-updates of one fwd+adj pass over all shots."""
        return self.grid.ncell * self.grid.nt * len(self.shots)


def _receivers_grid(n_side: int, step: int, first: int, z: int, npml: int):
    xs = first + step * np.arange(n_side)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    zr = np.full(X.size, z + npml, np.int32)
    return zr, (X.ravel() + npml).astype(np.int32), (Y.ravel() + npml).astype(np.int32)


def config1(nt: Optional[int] = None) -> Problem:
    """64^3 model, dx 10 m, 10-cell C-PML, dt 1 ms, nt 500, 10 Hz Ricker at
    (x, y, z) = (32, 32, 5), 32 x 32 receivers on z = 2; three flat layers
    vp 2000/2600/3200, vs = vp/1.732, rho = 310 vp^0.25; true model adds a
    +5 % Gaussian vp blob (sigma 6 cells) at the centre."""
    n, npml, dt, f0 = 64, 10, 1e-3, 10.0
    nt = nt or 500
    z = np.arange(n)[:, None, None] * np.ones((1, n, n))
    vp = np.where(z < n // 3, 2000.0, np.where(z < 2 * n // 3, 2600.0, 3200.0))
    vs = vp / 1.732
    rho = 310.0 * vp ** 0.25
    vp_true = vp * (1.0 + 0.05 * gaussian_blob((n, n, n), (n / 2, n / 2, n / 2), 6.0))
    rho_true = rho
    grid = Grid(n + 2 * npml, n + 2 * npml, n + 2 * npml, npml, nt, 10.0, 10.0, 10.0, dt, f0)
    zr, xr, yr = _receivers_grid(32, 2, 1, 2, npml)
    shots = [Shot(src=(5 + npml, 32 + npml, 32 + npml), z_rec=zr, x_rec=xr, y_rec=yr)]
    stf = ricker(f0, nt, dt)[None, :]
    return Problem("config1: 64^3, 1 shot, nt=%d" % nt, grid, shots, stf,
                   vp_true.astype(np.float32), vs.astype(np.float32), rho_true.astype(np.float32),
                   vp.astype(np.float32), vs.astype(np.float32), rho.astype(np.float32))


def config2(nt: Optional[int] = None, nshot: int = 16, seed: int = 2, n: int = 128) -> Problem:
    """128^3 model, dx 10 m, 12-cell C-PML, dt 0.8 ms, nt 2000, 16 Ricker
    8 Hz sources on a 4 x 4 surface grid, 64 x 64 receivers; 5 random layers
    vp in [1800, 4000] plus 8 Gaussian anomalies of +-8 % vp and +-10 % vs;
    initial model = truth smoothed with sigma 8 cells."""
    npml, dt, f0 = 12, 8e-4, 8.0
    nt = nt or 2000
    rng = np.random.default_rng(seed)
    bounds = np.sort(rng.choice(np.arange(8, n - 8), size=4, replace=False))
    vps = np.sort(rng.uniform(1800.0, 4000.0, size=5))
    zc = np.arange(n)
    vp1 = vps[np.searchsorted(bounds, zc, side="right")]
    vp = np.broadcast_to(vp1[:, None, None], (n, n, n)).astype(np.float64).copy()
    vs = vp / 1.732
    for _ in range(8):
        c = rng.uniform(0.2 * n, 0.8 * n, size=3)
        s = rng.uniform(0.04 * n, 0.1 * n)
        g = gaussian_blob((n, n, n), c, s)
        vp *= 1.0 + rng.choice([-1.0, 1.0]) * 0.08 * g
        vs *= 1.0 + rng.choice([-1.0, 1.0]) * 0.10 * g
    rho = 310.0 * vp ** 0.25
    vp, vs, rho = (a.astype(np.float32) for a in (vp, vs, rho))
    vp0, vs0, rho0 = smooth(vp, 8.0), smooth(vs, 8.0), smooth(rho, 8.0)
    N = n + 2 * npml
    grid = Grid(N, N, N, npml, nt, 10.0, 10.0, 10.0, dt, f0)
    side = int(round(np.sqrt(nshot)))
    pos = (np.arange(side) + 0.5) * (n / side)
    zr, xr, yr = _receivers_grid(64, max(n // 64, 1), max(n // 128, 0), 2, npml)
    shots = []
    for a in range(side):
        for b in range(side):
            shots.append(Shot(src=(4 + npml, int(pos[a]) + npml, int(pos[b]) + npml),
                              z_rec=zr, x_rec=xr, y_rec=yr))
    stf = np.tile(ricker(f0, nt, dt), (len(shots), 1))
    return Problem("config2: %d^3, %d shots, nt=%d" % (n, len(shots), nt), grid, shots, stf,
                   vp, vs, rho, vp0, vs0, rho0)


def small(nz=26, nx=30, ny=28, npml=6, nt=120, nshot=1, nrec=12, seed=0, dt=1e-3, f0=12.0,
          dx=10.0, dy=11.0, dz=9.0, contrast=0.05) -> Problem:
    """Small non-cubic problem for parity tests (sizes are padded sizes)."""
    rng = np.random.default_rng(seed)
    mz, mx, my = nz - 2 * npml, nx - 2 * npml, ny - 2 * npml
    z = np.arange(mz)[:, None, None] * np.ones((1, mx, my))
    vp = np.where(z < mz // 2, 2000.0, 2600.0) + 40.0 * rng.standard_normal((mz, mx, my))
    vs = vp / 1.732
    rho = 310.0 * vp ** 0.25
    vp_true = vp * (1.0 + contrast * gaussian_blob((mz, mx, my), (mz / 2, mx / 2, my / 2), 2.5))
    grid = Grid(nz, nx, ny, npml, nt, dz, dx, dy, dt, f0)
    shots = []
    for k in range(nshot):
        src = (npml + 2 + (k % 2), npml + 2 + (3 * k) % max(mx - 4, 1), npml + 3 + (5 * k) % max(my - 6, 1))
        zr = np.full(nrec, npml + 1, np.int32)
        xr = (npml + rng.integers(0, mx, nrec)).astype(np.int32)
        yr = (npml + rng.integers(0, my, nrec)).astype(np.int32)
        shots.append(Shot(src=src, z_rec=zr, x_rec=xr, y_rec=yr))
    stf = np.stack([ricker(f0 * (1.0 + 0.1 * k), nt, dt) for k in range(nshot)])
    return Problem("small", grid, shots, stf, vp_true.astype(np.float32), vs.astype(np.float32),
                   rho.astype(np.float32), vp.astype(np.float32), vs.astype(np.float32),
                   rho.astype(np.float32))


def config3(nt: Optional[int] = None, nshot: int = 4, seed: int = 3) -> Problem:
    """96^3 model (120^3 padded with a 12-cell C-PML), 4 shots, nt 4000: the
    differentiation and checkpointing configuration.  It names no spacing,
    time step or wavelet; those of config 2 are used (dx 10 m, dt 0.8 ms,
    8 Hz Ricker, random layers and anomalies, smoothed initial model)."""
    p = config2(nt=nt or 4000, nshot=nshot, seed=seed, n=96)
    p.name = "config3: 96^3, %d shots, nt=%d" % (len(p.shots), p.grid.nt)
    return p
