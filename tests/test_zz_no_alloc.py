"""The allocation-free misfit entry point (efwi_misfit_noalloc).

It exists for callers that cannot call cudaMalloc (device memory reserved up
front by another allocator, or a latency-critical path that cannot take
cudaMalloc's device-wide synchronisation).  Called twice in a row through
the C ABI, it must reproduce the misfit and adjoint source of the existing
gradient entry point (efwi_gradient), plain and windowed; an oversized
request must be rejected.  This file runs last so that a failure here comes
after every other test.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from helpers import fixture_engine, golden, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _ready():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _ptr(t):
    return C.c_void_p(t.data_ptr() if t is not None else 0)


@pytest.mark.parametrize("prefix,if_win", [("B_", False), ("C_", True)])
def test_noalloc_misfit_matches_gradient_entry_point(prefix, if_win):
    from efwi import _lib
    from efwi.engine import Propagator
    d = golden()
    g, shots, stf, lam, mu, rho = fixture_engine(prefix)
    P = Propagator(g, if_win=if_win)
    P.set_model(torch.from_numpy(lam), torch.from_numpy(mu), torch.from_numpy(rho))
    P.set_survey(shots, stf)
    obs = torch.from_numpy(d[prefix + "obs"]).cuda()
    syn = P.forward([0])
    J, _, _, _, res = P.gradient([0], obs, want_residual=True)
    sh = shots[0]
    win = [None, None, None]
    if if_win:
        win = [torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
               for a in (sh.win_start, sh.win_end, sh.weights)]
    L = _lib.lib()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        res2 = torch.full_like(obs, float("nan"))
        J2 = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        rc = L.efwi_misfit_noalloc(sh.nrec, g.nt, g.dt, int(if_win), _ptr(win[0]), _ptr(win[1]),
                                   _ptr(win[2]), sh.src_weight, _ptr(obs), _ptr(syn), _ptr(res2),
                                   _ptr(J2), stream)
        assert rc == _lib.EFWI_OK
        torch.cuda.synchronize()
        assert abs(J2.item() - J) <= 1e-6 * J
        assert rel_l2(res2.cpu(), res.cpu()) < 1e-6


def test_noalloc_rejects_requests_beyond_its_scratch():
    from efwi import _lib
    L = _lib.lib()
    t = torch.zeros(4, device="cuda")
    J = torch.zeros(1, dtype=torch.float64, device="cuda")
    # 3 * ceil(nt/32) * ceil(nrec/32) tiles > EFWI_NOALLOC_MAX_PARTIALS
    nrec, nt = 32 * 1024, 32 * 1024
    assert 3 * (nt // 32) * (nrec // 32) > _lib.NOALLOC_MAX_PARTIALS
    rc = L.efwi_misfit_noalloc(nrec, nt, 1e-3, 0, None, None, None, 1.0, _ptr(t), _ptr(t),
                               _ptr(t), _ptr(J), None)
    assert rc == _lib.EFWI_ERR_TOO_LARGE
