"""Host-side logic and the C-ABI library (CPU only, no compute calls)."""
import ctypes as C
import json
import os
import re
import threading

import numpy as np
import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    txt = open(os.path.join(ROOT, "include", "efwi.h")).read()
    return sorted(set(re.findall(r"\b(efwi_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from efwi import _lib
    L = _lib.lib()
    declared = _header_symbols()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(L, name), name
    assert sorted(_lib.exported_symbols()) == declared


def test_library_metadata_calls_without_gpu():
    from efwi import _lib
    L = _lib.lib()
    assert b"sm_100a" in L.efwi_version()
    names = _lib.kernel_names()
    assert "stress_fwd" in names and "rev_stress" in names


def test_create_rejects_bad_grid_without_touching_the_gpu():
    from efwi import _lib
    L = _lib.lib()
    g = _lib.EfwiGrid(10, 10, 10, 6, 100, 10., 10., 10., 1e-3, 10.)  # 2*npml > n
    h = C.c_void_p()
    rc = L.efwi_create(C.byref(g), C.byref(h))
    assert rc == _lib.EFWI_ERR_ARG
    assert b"invalid grid" in L.efwi_last_error(h)
    L.efwi_destroy(h)


def test_no_cpu_fallback():
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from efwi.engine import Grid, Propagator
    with pytest.raises(RuntimeError, match="CUDA device is required"):
        Propagator(Grid(20, 20, 20, 4, 10, 10., 10., 10., 1e-3, 10.))


# ------------------------------------------------------------------ configs
def _write_case(tmp_path, if_win=False, drop=None):
    import fwi_utils as ft
    para = str(tmp_path / "para.json")
    survey = str(tmp_path / "survey.json")
    data = str(tmp_path / "Data")
    ft.paraGen_3d(30, 32, 34, 10.0, 11.0, 12.0, 100, 1e-3, 10.0, 6, para, survey, data,
                  if_win=if_win)
    zs = np.array([[2, 2], [2, 2]])
    xs = np.array([[3, 4], [5, 6]])
    ys = np.array([[7, 8], [9, 10]])
    zr = np.array([1, 1, 1])
    xr = np.array([2, 3, 4])
    yr = np.array([5, 6, 7])
    ft.surveyGen_3d(zs, xs, ys, zr, xr, yr, survey)
    if drop:
        d = json.load(open(para))
        d.pop(drop)
        json.dump(d, open(para, "w"))
    return para, survey, data


def test_para_and_survey_round_trip(tmp_path):
    from efwi import config
    para, survey, data = _write_case(tmp_path)
    p = config.read_para(para)
    assert (p.grid.nz, p.grid.nx, p.grid.ny, p.grid.npml, p.grid.nt) == (30, 32, 34, 6, 100)
    assert p.data_dir_name == data and os.path.isdir(data)
    shots = config.read_survey(p.survey_fname, p.grid.npml)
    assert len(shots) == 4
    # shot i = element (i % 2, i // 2); coordinates get + nPml
    assert tuple(shots[1].src) == (2 + 6, 5 + 6, 9 + 6)
    assert tuple(shots[2].src) == (2 + 6, 4 + 6, 8 + 6)
    assert list(shots[0].x_rec) == [8, 9, 10]


def test_missing_para_key_raises(tmp_path):
    from efwi import config
    para, _, _ = _write_case(tmp_path, drop="dt")
    with pytest.raises(config.ConfigError, match="dt"):
        config.read_para(para)


def test_missing_files_raise(tmp_path):
    from efwi import config
    with pytest.raises(config.ConfigError, match="cannot open"):
        config.read_para(str(tmp_path / "nope.json"))
    with pytest.raises(config.ConfigError, match="file reading error"):
        config.read_shot_data(str(tmp_path), 3, 4, 10)


def test_windowed_survey_requires_windows(tmp_path):
    from efwi import config
    para, survey, _ = _write_case(tmp_path, if_win=True)
    p = config.read_para(para)
    assert p.if_win
    with pytest.raises(config.ConfigError, match="win_start"):
        config.read_survey(survey, p.grid.npml, if_win=True)


def test_shot_data_round_trip(tmp_path):
    from efwi import config
    a = np.random.default_rng(0).standard_normal((3, 5, 7)).astype(np.float32)
    config.write_shot_data(str(tmp_path), 4, a)
    raw = np.fromfile(tmp_path / "Shot_y4.bin", dtype=np.float32).reshape(5, 7)
    np.testing.assert_array_equal(raw, a[1])
    np.testing.assert_array_equal(config.read_shot_data(str(tmp_path), 4, 5, 7), a)


def test_shard_split_matches_reference_rule():
    import FWI_ops_3d as F
    # linspace(0, n, ngpu+1) truncated (Torch_Fwi.cpp:53-54,74-76)
    assert F._shards(list(range(5)), 2) == [[0, 1], [2, 3, 4]]
    assert F._shards(list(range(16)), 3) == [[0, 1, 2, 3, 4], [5, 6, 7, 8, 9], [10, 11, 12, 13, 14, 15]]
    assert sum(F._shards(list(range(7)), 7), []) == list(range(7))


def test_ngpu_above_shot_count_raises():
    import FWI_ops_3d as F
    with pytest.raises(ValueError, match="number of GPUs"):
        F.fwi_ops.backward(torch.zeros(1), torch.zeros(1), torch.zeros(1), torch.zeros(1, 1), 3,
                           torch.tensor([0, 1], dtype=torch.int32), "unused.json")


# ---------------------------------------------------------------- fwi_utils
def test_padding_replicates_edges():
    import fwi_utils as ft
    v = torch.arange(2 * 3 * 4, dtype=torch.float32).reshape(2, 3, 4)
    a, b, c = ft.padding_3d(v, v, v, 2, 3, 4, 2)
    assert a.shape == (6, 7, 8)
    np.testing.assert_array_equal(a.numpy(), np.pad(v.numpy(), 2, mode="edge"))


def test_padding_is_differentiable():
    import fwi_utils as ft
    v = torch.rand(2, 3, 4, requires_grad=True)
    a, _, _ = ft.padding_3d(v, v, v, 2, 3, 4, 1)
    a.sum().backward()
    # every cell gets one from itself plus the copies made by the padding
    assert v.grad.sum().item() == pytest.approx(a.numel())


def test_source_gene_is_integrated_ricker():
    import fwi_utils as ft
    f, n, dt = 4.5, 400, 2.5e-3
    s = ft.sourceGene(f, n, dt)
    e = np.pi ** 2 * f * f
    ref = np.zeros(n)
    for it in range(n):
        t = dt * it - 1.2 / f
        ref[it] = (1 - 2 * e * t * t) * np.exp(-e * t * t)
    for it in range(1, n):
        ref[it] += ref[it - 1]
    np.testing.assert_allclose(s, ref * dt, rtol=1e-12, atol=1e-15)


def test_fwi3d_default_mask_is_full_size():
    import FWI_ops_3d as F
    vp = torch.full((4, 5, 6), 2000.0)
    m = F.FWI_3d(vp, vp / 2, vp, torch.zeros(1, 10), {"nz": 4, "nx": 5, "ny": 6, "nPml": 2,
                                                       "para_fname": "x"})
    assert tuple(m.Mask.shape) == (8, 9, 10)
