"""Learned gradient preconditioner for vp inversion (no reference counterpart).

* Training data (pseudo-Hessian pairs): on seeded random layered + anomaly
  models, the vp gradient g, the current model and the source illumination
  (diagonal pseudo-Hessian of Shin et al. 2001, efwi_illumination) are the
  inputs; the target is the gradient preconditioned by a random-probe
  estimate of the Gauss-Newton diagonal, diag(J^T J) ~ mean_k (J^T w_k)^2
  over white Rademacher probes w_k in data space (efwi_adjoint) -- the
  probing estimator of Bekas, Kokiopoulou & Saad (2007) applied to J^T J.
* The CNN (efwi.cnn.Preconditioner, BF16 tensor-core convolutions) maps the
  cheap inputs to the expensive direction.
* L-BFGS with the learned step (net_mode "step"): each iteration first
  tries the CNN's direction under a backtracking Armijo line search; if the
  line search rejects it, the plain L-BFGS direction is used (and is itself
  line searched).  The curvature pairs of accepted steps feed the L-BFGS
  memory either way.  The plain method is the same loop without the CNN.
* net_mode "h0": the CNN, made homogeneous in its gradient input, is the
  initial inverse Hessian of the two-loop recursion (Nocedal & Wright 2006,
  Algorithm 7.4, with H0 = gamma N instead of gamma I; gamma = s'y / y'N(y)
  along the newest pair), so the learned map preconditions the quasi-Newton
  step instead of replacing it; the identity-H0 direction is the fallback
  when the line search rejects the preconditioned one.

The model is vp on the model grid; vs and rho stay at their initial values,
as in the reference's inversion drivers, which update vp only
(3D_inversion_adam.py).  lambda = (vp^2 - 2 vs^2) rho and mu = vs^2 rho on the
padded grid (FWI_ops_3d.py:86-94 with replicate padding, fwi_utils.py:9-20).
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass
from typing import Dict, List, Optional

import numpy as np
import torch
import torch.nn.functional as F

from . import synthetic
from .autograd import misfit as exact_misfit
from .engine import Grid, Propagator, Shot


def layered_problem(n: int = 40, npml: int = 8, nt: int = 500, shots_side: int = 2,
                    seed: int = 0, dx: float = 10.0, dt: float = 8e-4, f0: float = 8.0,
                    smooth_sigma: float = 6.0) -> synthetic.Problem:
    """Random layered model with Gaussian anomalies (vp in [1800, 4000] m/s,
    +-8 % vp and +-10 % vs anomalies, rho = 310 vp^0.25); the initial model
    is the truth smoothed with a Gaussian of `smooth_sigma` cells.  Sources
    on a shots_side^2 surface grid, receivers every 2 cells at depth 2."""
    rng = np.random.default_rng(seed)
    nl = int(rng.integers(3, 6))
    bounds = np.sort(rng.choice(np.arange(4, n - 4), size=nl - 1, replace=False))
    vps = np.sort(rng.uniform(1800.0, 4000.0, size=nl))
    vp1 = vps[np.searchsorted(bounds, np.arange(n), side="right")]
    vp = np.broadcast_to(vp1[:, None, None], (n, n, n)).astype(np.float64).copy()
    vs = vp / 1.732
    for _ in range(int(rng.integers(3, 9))):
        c = rng.uniform(0.2 * n, 0.8 * n, size=3)
        s = rng.uniform(0.05 * n, 0.12 * n)
        g = synthetic.gaussian_blob((n, n, n), c, s)
        vp *= 1.0 + rng.choice([-1.0, 1.0]) * 0.08 * g
        vs *= 1.0 + rng.choice([-1.0, 1.0]) * 0.10 * g
    rho = 310.0 * vp ** 0.25
    vp, vs, rho = (a.astype(np.float32) for a in (vp, vs, rho))
    vp0, vs0, rho0 = (synthetic.smooth(a, smooth_sigma) for a in (vp, vs, rho))
    N = n + 2 * npml
    grid = Grid(N, N, N, npml, nt, dx, dx, dx, dt, f0)
    xs = np.arange(1, n - 1, 2)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    zr = np.full(X.size, 2 + npml, np.int32)
    xr, yr = (X.ravel() + npml).astype(np.int32), (Y.ravel() + npml).astype(np.int32)
    pos = (np.arange(shots_side) + 0.5) * (n / shots_side)
    shots = [Shot(src=(3 + npml, int(a) + npml, int(b) + npml), z_rec=zr, x_rec=xr, y_rec=yr)
             for a in pos for b in pos]
    stf = np.tile(synthetic.ricker(f0, nt, dt), (len(shots), 1))
    return synthetic.Problem(f"layered {n}^3 seed {seed}", grid, shots, stf, vp, vs, rho,
                             vp0, vs0, rho0)


class VpObjective:
    """Misfit of vp (model grid) with vs and rho fixed, on one GPU."""

    def __init__(self, prob: synthetic.Problem, device=None, mode: str = "exact",
                 obs: Optional[torch.Tensor] = None, checkpoint_gib: float = 8.0):
        self.prob = prob
        self.mode = mode
        self.P = Propagator(prob.grid, device=device)
        self.dev = self.P.device
        self.P.set_checkpoint_budget(int(checkpoint_gib * (1 << 30)))
        self.P.set_survey(prob.shots, prob.stf)
        self.ids = list(range(len(prob.shots)))
        if obs is None:
            lt, mt, rt = prob.params("true")
            self.P.set_model(torch.from_numpy(lt), torch.from_numpy(mt), torch.from_numpy(rt))
            obs = self.P.forward(self.ids)
        self.obs = obs
        npml = prob.grid.npml
        self.npml = npml
        self.vs_p = self._pad(torch.from_numpy(prob.vs_init).to(self.dev))
        self.rho_p = self._pad(torch.from_numpy(prob.rho_init).to(self.dev)) / 1e3
        self.vp_true = torch.from_numpy(prob.vp_true).to(self.dev)
        self.evals = 0

    def _pad(self, v: torch.Tensor) -> torch.Tensor:
        p = self.npml
        return F.pad(v[None, None], (p, p, p, p, p, p), mode="replicate")[0, 0]

    def params(self, vp: torch.Tensor):
        vp_p = self._pad(vp)
        lam = (vp_p * vp_p - 2.0 * self.vs_p * self.vs_p) * self.rho_p
        mu = self.vs_p * self.vs_p * self.rho_p
        return lam, mu, self.rho_p

    def value_and_grad(self, vp: torch.Tensor):
        """J(vp) and dJ/dvp (model grid)."""
        self.evals += 1
        v = vp.detach().clone().requires_grad_(True)
        lam, mu, rho = self.params(v)
        if self.mode == "exact":
            J = exact_misfit(lam, mu, rho, self.P, self.ids, self.obs)
            J.backward()
            return float(J.item()), v.grad.detach()
        self.P.set_model(lam.detach(), mu.detach(), rho)
        Jv, gl, gm, gr = self.P.gradient(self.ids, self.obs, mode="reference")
        (g,) = torch.autograd.grad(lam, v, grad_outputs=gl)
        return float(Jv), g.detach()

    def value(self, vp: torch.Tensor) -> float:
        self.evals += 1
        lam, mu, rho = self.params(vp.detach())
        self.P.set_model(lam, mu, rho)
        return float(self.P.misfit(self.ids, self.obs))

    def _to_vp(self, vp: torch.Tensor, g_lam: torch.Tensor, square: bool = False) -> torch.Tensor:
        """Chain a lambda-space quantity to vp (dlambda/dvp = 2 vp rho): a
        gradient through the padding, or (square) a diagonal on the model
        grid."""
        if square:
            d = 2.0 * self._pad(vp) * self.rho_p
            p = self.npml
            return (g_lam * d * d)[p:-p, p:-p, p:-p]
        v = vp.detach().clone().requires_grad_(True)
        lam, _, _ = self.params(v)
        (g,) = torch.autograd.grad(lam, v, grad_outputs=g_lam)
        return g

    def illumination(self, vp: torch.Tensor) -> torch.Tensor:
        """Shin pseudo-Hessian diagonal of vp (model grid)."""
        lam, mu, rho = self.params(vp.detach())
        self.P.set_model(lam, mu, rho)
        hl, _, _ = self.P.illumination(self.ids)
        return self._to_vp(vp, hl, square=True)

    def probe_diagonal(self, vp: torch.Tensor, nprobe: int = 4, seed: int = 0) -> torch.Tensor:
        """mean_k ((J^T w_k)_vp)^2 over Rademacher probes w_k."""
        lam, mu, rho = self.params(vp.detach())
        self.P.set_model(lam, mu, rho)
        gen = torch.Generator(device=self.dev).manual_seed(seed)
        acc = torch.zeros_like(vp)
        for _ in range(nprobe):
            w = torch.randint(0, 2, self.obs.shape, generator=gen, device=self.dev,
                              dtype=torch.int32).float() * 2.0 - 1.0
            gl, _, _ = self.P.adjoint(self.ids, w)
            g = self._to_vp(vp, gl)
            acc += g * g
        return acc / nprobe

    def close(self):
        self.P.close()


def features(g: torch.Tensor, vp: torch.Tensor, illum: torch.Tensor) -> torch.Tensor:
    """CNN inputs [3, D, H, W]: normalised gradient, model and log-illumination."""
    gn = g / (g.abs().max() + 1e-30)
    vn = (vp - vp.mean()) / (vp.std() + 1e-6)
    il = torch.log10(illum / (illum.max() + 1e-30) + 1e-6) / 6.0 + 1.0
    return torch.stack([gn, vn, il]).float()


def target_direction(g: torch.Tensor, diag: torch.Tensor, eps: float = 1e-3) -> torch.Tensor:
    d = g / (diag + eps * diag.max())
    return d / (d.abs().max() + 1e-30)


def make_pairs(n_pairs: int = 200, n: int = 40, nt: int = 500, nprobe: int = 4, seed0: int = 1000,
               device=None, mode: str = "exact", log=None) -> List[Dict[str, torch.Tensor]]:
    """(features, target) pairs on seeded random layered + anomaly models."""
    out = []
    for k in range(n_pairs):
        prob = layered_problem(n=n, nt=nt, seed=seed0 + k)
        obj = VpObjective(prob, device=device, mode=mode)
        vp = torch.from_numpy(prob.vp_init).to(obj.dev)
        _, g = obj.value_and_grad(vp)
        il = obj.illumination(vp)
        dg = obj.probe_diagonal(vp, nprobe=nprobe, seed=seed0 + k)
        out.append({"x": features(g, vp, il), "y": target_direction(g, dg)})
        obj.close()
        if log:
            log(f"pair {k + 1}/{n_pairs}")
    return out


def _cosine_loss(pred: torch.Tensor, y: torch.Tensor) -> torch.Tensor:
    """1 - cos(pred, y) over the whole volume: only the direction counts (the
    L-BFGS recursion rescales the map's output), and every cell weighs by its
    share of the norm rather than by its size relative to the largest entry
    (a mean squared error of max-normalised directions is near its floor
    for any output close to zero)."""
    p, t = pred.reshape(-1), y.reshape(-1)
    return 1.0 - torch.dot(p, t) / (torch.linalg.vector_norm(p) * torch.linalg.vector_norm(t) + 1e-30)


def train(net, pairs, epochs: int = 20, lr: float = 2e-3, seed: int = 0, log=None) -> List[float]:
    """Adam on one minus the cosine between the network's output and the
    target direction."""
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    g = torch.Generator().manual_seed(seed)
    hist = []
    for ep in range(epochs):
        order = torch.randperm(len(pairs), generator=g).tolist()
        tot = 0.0
        for i in order:
            opt.zero_grad()
            pred = net(pairs[i]["x"])
            loss = _cosine_loss(pred, pairs[i]["y"])
            loss.backward()
            opt.step()
            tot += loss.item()
        hist.append(tot / len(pairs))
        if log:
            log(f"epoch {ep + 1}: loss {hist[-1]:.4e}")
    return hist


# ------------------------------------------------------------------ L-BFGS
@dataclass
class LbfgsResult:
    misfit: List[float]
    seconds: List[float]
    model_rel_l2: List[float]
    learned_accepted: int
    evals: int


def _sync(dev) -> None:
    if torch.device(dev).type == "cuda":
        torch.cuda.synchronize(dev)


def _dot(a: torch.Tensor, b: torch.Tensor) -> float:
    """Inner product in FP64, so that the recursion does not depend on the
    scale of the misfit (squares of small FP32 gradient entries underflow
    FP32, and sums over millions of cells lose digits)."""
    return float(torch.sum(a.double() * b.double()))


def lbfgs(obj: VpObjective, vp0: torch.Tensor, iters: int = 20, memory: int = 10,
          net=None, first_step: float = 20.0, c1: float = 1e-4, max_trials: int = 12,
          max_expand: int = 3, learned_trials: int = 4,
          stop_misfit: Optional[float] = None, bounds=(1000.0, 6000.0), log=None,
          net_mode: str = "step") -> LbfgsResult:
    """L-BFGS on vp with an Armijo line search -- backtracking by halves, or
    doubling (up to max_expand times) while the misfit keeps falling when
    the unit step is accepted at once; trial points cost a forward
    modelling, the accepted point a gradient.  With `net`,
    each iteration first tries the CNN's direction (scaled so that its
    largest vp change is the previous accepted step's, at most
    `learned_trials` halvings); the plain L-BFGS direction is the fallback
    when that line search fails.  `first_step`
    (m/s) scales the first plain step, like the reference's Adam learning
    rate of 20 m/s (3D_inversion_adam.py).

    net_mode "h0" uses `net` as the initial inverse Hessian of the two-loop
    recursion instead (module docstring); `learned_accepted` then counts the
    iterations whose preconditioned direction was accepted."""
    if net_mode not in ("step", "h0"):
        raise ValueError(f"net_mode must be 'step' or 'h0', not {net_mode!r}")
    _sync(obj.dev)
    t0 = time.perf_counter()
    vp = vp0.clone()
    J, g = obj.value_and_grad(vp)
    S, Y = [], []
    res = LbfgsResult([J], [0.0], [_rel(vp, obj.vp_true)], 0, obj.evals)
    last_dmax = first_step
    illum = obj.illumination(vp) if net is not None else None

    def learned_map(q):
        """The CNN applied to q as a gradient, scaled back by q's largest
        entry, so that N(c q) = c N(q) for c > 0."""
        with torch.no_grad():
            return net(features(q, vp, illum)).to(q.dtype) * q.abs().max()

    def two_loop(q, h0=None):
        q = q.clone()
        al = []
        for s, y in reversed(list(zip(S, Y))):
            rho = 1.0 / _dot(y, s)
            a = rho * _dot(s, q)
            q -= a * y
            al.append((rho, a))
        if h0 is not None:
            nq = h0(q)
            if S:
                yn = _dot(Y[-1], h0(Y[-1]))
                if not float(yn) > 0:
                    return None  # the map is not positive along y: no learned H0
                r = (_dot(S[-1], Y[-1]) / yn) * nq
            else:
                r = nq * (first_step / (nq.abs().max() + 1e-30))
        elif S:
            gamma = _dot(S[-1], Y[-1]) / _dot(Y[-1], Y[-1])
            r = gamma * q
        else:
            r = q * (first_step / (q.abs().max() + 1e-30))
        for (s, y), (rho, a) in zip(zip(S, Y), reversed(al)):
            b = rho * _dot(y, r)
            r += s * (a - b)
        return -r

    def search(d, J, g, trials):
        gd = _dot(g, d)
        if not gd < 0:
            return None
        alpha = 1.0
        for _ in range(trials):
            vn = torch.clamp(vp + alpha * d, *bounds)
            Jn = obj.value(vn)  # trial points need the misfit only
            if Jn <= J + c1 * alpha * gd:
                if alpha == 1.0:
                    # accepted at once: extrapolate while the misfit keeps falling
                    for _ in range(max_expand):
                        vx = torch.clamp(vp + 2.0 * alpha * d, *bounds)
                        Jx = obj.value(vx)
                        if not (Jx < Jn and Jx <= J + c1 * 2.0 * alpha * gd):
                            break
                        alpha, vn, Jn = 2.0 * alpha, vx, Jx
                Jn, gn = obj.value_and_grad(vn)
                return vn, Jn, gn
            alpha *= 0.5
        return None

    for it in range(iters):
        step = None
        if net is not None and net_mode == "h0":
            d = two_loop(g, learned_map)
            step = search(d, J, g, max_trials) if d is not None else None
            if step is not None:
                res.learned_accepted += 1
        elif net is not None:
            with torch.no_grad():
                dl = -net(features(g, vp, illum))
            dl = dl * (last_dmax / (dl.abs().max() + 1e-30))
            step = search(dl, J, g, learned_trials)
            if step is not None:
                res.learned_accepted += 1
        if step is None:
            step = search(two_loop(g), J, g, max_trials)
        if step is None:
            break
        vn, Jn, gn = step
        s, y = vn - vp, gn - g
        if _dot(s, y) > 1e-12 * _dot(y, y):
            S.append(s)
            Y.append(y)
            if len(S) > memory:
                S.pop(0)
                Y.pop(0)
        last_dmax = float(s.abs().max())
        vp, J, g = vn, Jn, gn
        _sync(obj.dev)
        res.misfit.append(J)
        res.seconds.append(time.perf_counter() - t0)
        res.model_rel_l2.append(_rel(vp, obj.vp_true))
        res.evals = obj.evals
        if log:
            log(f"iter {it + 1}: misfit {J:.6e}, {res.seconds[-1]:.1f} s, "
                f"model rel-L2 {res.model_rel_l2[-1]:.4e}")
        if stop_misfit is not None and J <= stop_misfit:
            break
    res.evals = obj.evals  # trial points of a failed last search included
    return res


def _rel(a, b) -> float:
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
