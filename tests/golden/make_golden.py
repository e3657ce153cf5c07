"""Generates tests/golden/ref_small.npz from the reference's own kernels.

The reference has no tests or golden vectors for this path.  These fixtures
are produced by running the reference's kernel sources (Ops/FWI/Src_3d,
compiled for the CPU into oracle/_ref/libefwi_ref.so by oracle/Makefile) on
small seeded problems.  They pin the FP64 oracle (tests/test_oracle.py) and
the CUDA engine (tests/test_parity_gpu.py).

Run from the repository root where the reference tree is present:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "efwi-3d_b200"), os.path.dirname(HERE)]

import oracle  # noqa: E402
from efwi import synthetic  # noqa: E402
from helpers import case_of  # noqa: E402


def pack(prefix, p, out, if_win=False):
    g = p.grid
    lam, mu, rho = p.params("init")
    lt, mt, rt = p.params("true")
    out[prefix + "grid_i"] = np.array([g.nz, g.nx, g.ny, g.npml, g.nt], np.int32)
    out[prefix + "grid_f"] = np.array([g.dz, g.dx, g.dy, g.dt, g.f0], np.float32)
    out[prefix + "lam"], out[prefix + "mu"], out[prefix + "rho"] = lam, mu, rho
    out[prefix + "lam_true"], out[prefix + "mu_true"], out[prefix + "rho_true"] = lt, mt, rt
    out[prefix + "src"] = np.array([s.src for s in p.shots], np.int32)
    out[prefix + "rec"] = np.stack([np.stack([s.z_rec, s.x_rec, s.y_rec]) for s in p.shots]).astype(np.int32)
    out[prefix + "stf"] = p.stf.astype(np.float32)
    if if_win:
        out[prefix + "win"] = np.stack([np.stack([s.win_start, s.win_end, s.weights]) for s in p.shots]).astype(np.float32)
        out[prefix + "src_weight"] = np.array([s.src_weight for s in p.shots], np.float32)


def main():
    oracle.build()
    R = oracle.ref()
    out = {}
    # A: forward traces, two shots, non-cubic grid.
    pa = synthetic.small(nz=26, nx=30, ny=28, npml=6, nt=150, nshot=2, nrec=16, seed=11)
    pack("A_", pa, out)
    tr = R.forward(case_of(pa, "init", np.float32))
    out["A_traces"] = np.concatenate([t.ravel() for t in tr]).astype(np.float32)
    # B: reference gradient, one shot, observed data from the true model.
    pb = synthetic.small(nz=22, nx=24, ny=20, npml=5, nt=110, nshot=1, nrec=12, seed=5,
                         contrast=0.08)
    pack("B_", pb, out)
    obs = R.forward(case_of(pb, "true", np.float32))
    J, gl, gm, gr, res = R.gradient(case_of(pb, "init", np.float32), obs)
    out["B_obs"] = np.concatenate([o.ravel() for o in obs]).astype(np.float32)
    out["B_misfit"] = np.array([J])
    out["B_glam"], out["B_gmu"], out["B_grho"] = gl, gm, gr
    out["B_res"] = np.concatenate([r.ravel() for r in res]).astype(np.float32)
    # C: windowed misfit (if_win) with per-trace windows and weights.
    pc = synthetic.small(nz=22, nx=24, ny=20, npml=5, nt=110, nshot=1, nrec=12, seed=7,
                         contrast=0.08)
    rng = np.random.default_rng(3)
    T = pc.grid.nt * pc.grid.dt
    for s in pc.shots:
        s.win_start = rng.uniform(0.0, 0.3 * T, s.nrec).astype(np.float32)
        s.win_end = rng.uniform(0.6 * T, 1.1 * T, s.nrec).astype(np.float32)
        s.win_end[0] = s.win_start[0]          # zero-length window: trace left untouched
        s.weights = rng.uniform(0.5, 1.5, s.nrec).astype(np.float32)
        s.src_weight = 0.75
    pack("C_", pc, out, if_win=True)
    obs = R.forward(case_of(pc, "true", np.float32))
    J, gl, gm, gr, res = R.gradient(case_of(pc, "init", np.float32, if_win=True), obs, if_win=True)
    out["C_obs"] = np.concatenate([o.ravel() for o in obs]).astype(np.float32)
    out["C_misfit"] = np.array([J])
    out["C_glam"], out["C_gmu"], out["C_grho"] = gl, gm, gr
    out["C_res"] = np.concatenate([r.ravel() for r in res]).astype(np.float32)
    # D: C-PML profiles and the source taper.
    prof = []
    for (n, npml, dh, f0, dt) in [(84, 10, 10.0, 10.0, 1e-3), (152, 12, 10.0, 8.0, 8e-4),
                                  (30, 6, 11.0, 12.0, 1e-3)]:
        prof.append(R.cpml(n, npml, dh, f0, dt).ravel())
    out["D_cpml_args"] = np.array([[84, 10, 10.0, 10.0, 1e-3], [152, 12, 10.0, 8.0, 8e-4],
                                   [30, 6, 11.0, 12.0, 1e-3]], np.float64)
    out["D_cpml"] = np.concatenate(prof).astype(np.float32)
    stf = synthetic.ricker(10.0, 500, 1e-3)
    out["D_stf"] = stf
    out["D_stf_tapered"] = R.taper_stf(stf, 1e-3)
    np.savez_compressed(os.path.join(HERE, "ref_small.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_small.npz"))


if __name__ == "__main__":
    main()
