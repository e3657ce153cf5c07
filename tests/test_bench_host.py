"""Host-side pieces of the benchmark and the preconditioner (no GPU): the
byte accounting behind the roofline figures, the window workload's
geometry, and the CNN's channels-last layout."""
import os
import sys

import numpy as np
import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402
from efwi import synthetic  # noqa: E402


@pytest.mark.parametrize("n,npml,per_cell", [(64, 10, 473.5), (128, 12, 442.5), (96, 12, 458.7)])
def test_gradient_step_bytes_per_padded_cell(n, npml, per_cell):
    """B_g = 3 (120 N + 48 S) + 24 N_int per step, per padded cell: 473.5 B
    (64^3 model, C-PML 10), 442.5 B (128^3, 12), 458.7 B (96^3, 12)."""
    m = n + 2 * npml
    g = synthetic.Grid(m, m, m, npml, 10, 10.0, 10.0, 10.0, 1e-3, 10.0)
    b = bench.algorithmic_step_bytes(g, n ** 3) / g.ncell
    assert abs(b - per_cell) < 0.1


def test_kernel_bytes_add_up_to_the_forward_and_reverse_sweeps():
    """Per shot-step the forward kernels move B_f = 120 N + 48 S; the two
    fused reverse kernels move 264 N + 72 S (reverse + adjoint sweeps)."""
    m = 152
    g = synthetic.Grid(m, m, m, 12, 10, 10.0, 10.0, 10.0, 1e-3, 10.0)
    kb = bench.kernel_bytes(g)
    N = g.ncell
    S = 2 * g.npml * 3 * m * m
    assert kb["stress_fwd"] + kb["velocity_fwd"] == 120 * N + 48 * S
    assert kb["rev_velocity"] + kb["rev_stress"] == 264 * N + 72 * S


def test_window_workload_geometry():
    """64 windows of lateral extent 96-192 cells plus C-PML, inside the
    256 x 256 x 160 model; each shot's source and receivers inside its own
    window."""
    grid, shots, stf, (vp, vs, rho), wins = bench.config4(nt=50)
    assert len(shots) == len(wins) == 64
    assert (grid.nz, grid.nx, grid.ny) == (184, 280, 280)
    for s, (x0, y0, nxw, nyw) in zip(shots, wins):
        L = nxw - 2 * grid.npml
        assert 96 <= L <= 192 and nxw == nyw
        assert 0 <= x0 and x0 + nxw <= grid.nx and 0 <= y0 and y0 + nyw <= grid.ny
        assert x0 + 2 <= s.src[1] <= x0 + nxw - 3 and y0 + 2 <= s.src[2] <= y0 + nyw - 3
        assert (s.x_rec >= x0).all() and (s.x_rec < x0 + nxw).all()
        assert (s.y_rec >= y0).all() and (s.y_rec < y0 + nyw).all()
    assert stf.shape == (64, 50)
    assert vp.shape == (160, 256, 256)


def test_channels_last_layout_pads_to_sixteen():
    from efwi.cnn import to_channels_last
    f = torch.arange(3 * 2 * 3 * 4, dtype=torch.float32).reshape(3, 2, 3, 4)
    x = to_channels_last(f)
    assert x.shape == (2, 3, 4, 16) and x.dtype == torch.bfloat16
    assert torch.equal(x[..., :3].float(), f.permute(1, 2, 3, 0).to(torch.bfloat16).float())
    assert float(x[..., 3:].abs().max()) == 0.0


def test_preconditioner_weights_respect_the_padded_channels():
    """The first layer reads only the real input channels and the last
    writes only output channel 0."""
    from efwi.cnn import Preconditioner
    net = Preconditioner(cin=3, seed=0)
    assert float(net.w[0].detach()[:, :, 3:].abs().max()) == 0.0
    assert float(net.w[-1].detach()[:, 1:, :].abs().max()) == 0.0
    assert len(net.w) == 4 and tuple(net.w[1].shape) == (27, 16, 16)
