"""Torch-facing wrapper of the C-ABI engine.

A :class:`Propagator` owns one engine handle on one CUDA device: the grid
and C-PML coefficients, the resident model (lambda, mu, buoyancy), the
survey, and the HBM workspace, all reused across calls.  Torch provides the
device memory and the stream; every operation runs in libefwi.so.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import EfwiGrid, EfwiShot, check, lib


@dataclass
class Grid:
    """Padded grid and time axis (the para JSON fields, Parameter.cpp:39-104)."""
    nz: int
    nx: int
    ny: int
    npml: int
    nt: int
    dz: float
    dx: float
    dy: float
    dt: float
    f0: float

    @property
    def shape(self):
        return (self.nz, self.nx, self.ny)

    @property
    def ncell(self) -> int:
        return self.nz * self.nx * self.ny


@dataclass
class Shot:
    """One shot on the padded grid (indices already include npml)."""
    src: Sequence[int]                      # (z, x, y)
    z_rec: np.ndarray
    x_rec: np.ndarray
    y_rec: np.ndarray
    win_start: Optional[np.ndarray] = None  # seconds, windowed misfit only
    win_end: Optional[np.ndarray] = None
    weights: Optional[np.ndarray] = None
    src_weight: float = 1.0

    @property
    def nrec(self) -> int:
        return int(len(self.z_rec))


def _f32_dev(t, device) -> torch.Tensor:
    t = torch.as_tensor(t)
    return t.to(device=device, dtype=torch.float32).contiguous()


class Propagator:
    """Elastic forward/adjoint engine for one grid on one GPU."""

    def __init__(self, grid: Grid, device=None, if_win: bool = False, tile_bx: int = 4,
                 zchunk: int = 8, max_batch: int = 4):
        if not torch.cuda.is_available():
            raise RuntimeError("efwi: a CUDA device is required (there is no CPU path)")
        self.grid = grid
        self.device = torch.device(device if device is not None else "cuda", )
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self._L = lib()
        g = EfwiGrid(grid.nz, grid.nx, grid.ny, grid.npml, grid.nt, grid.dz, grid.dx, grid.dy,
                     grid.dt, grid.f0)
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            rc = self._L.efwi_create(C.byref(g), C.byref(h))
        self._h = h
        check(h, rc)
        self.shots: List[Shot] = []
        self.set_options(if_win=if_win, tile_bx=tile_bx, zchunk=zchunk, max_batch=max_batch)
        self.lanes = 2  # the engine's default
        self._model_version = None

    # ------------------------------------------------------------------ setup
    def close(self) -> None:
        if getattr(self, "_h", None):
            with torch.cuda.device(self.device):
                self._L.efwi_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def set_options(self, if_win: bool = False, tile_bx: int = 0, zchunk: int = 0,
                    max_batch: int = 0) -> None:
        self.if_win = bool(if_win)
        check(self._h, self._L.efwi_set_options(self._h, int(if_win), int(tile_bx), int(zchunk),
                                                int(max_batch)))

    def set_graphs(self, on: bool) -> None:
        """Time loops as CUDA graphs replayed across shots and calls (default
        on); off launches every kernel from the host (same results)."""
        check(self._h, self._L.efwi_set_graphs(self._h, int(bool(on))))

    def set_variant(self, variant: int) -> None:
        """1: TMA-staged stencil planes (default); 0: L1-served stencils."""
        check(self._h, self._L.efwi_set_variant(self._h, int(variant)))

    def set_tuning(self, fwd_cfg: int = 0, zchunk_fwd: int = 0, rev_cfg: int = 0,
                   zchunk_rev: int = 0) -> None:
        """Launch configuration of the TMA kernels (see efwi_set_tuning)."""
        check(self._h, self._L.efwi_set_tuning(self._h, int(fwd_cfg), int(zchunk_fwd),
                                               int(rev_cfg), int(zchunk_rev)))
        self.tuning = (fwd_cfg, zchunk_fwd, rev_cfg, zchunk_rev)

    def set_lanes(self, lanes: int) -> None:
        """Shots of a reference-mode misfit/gradient call that run
        concurrently, each lane with its own workspace and stream (1-8,
        default 2; efwi_set_lanes)."""
        check(self._h, self._L.efwi_set_lanes(self._h, int(lanes)))
        self.lanes = int(lanes)

    def set_nt_limit(self, nt_limit: int) -> None:
        check(self._h, self._L.efwi_set_nt_limit(self._h, int(nt_limit)))

    def set_model(self, lam, mu, rho) -> None:
        """lambda, mu, rho on the padded grid, [nz][nx][ny] (any device)."""
        g = self.grid
        ts = [_f32_dev(t, self.device) for t in (lam, mu, rho)]
        for t in ts:
            if tuple(t.shape) != g.shape:
                raise ValueError(f"model shape {tuple(t.shape)} != grid {g.shape}")
        with torch.cuda.device(self.device):
            rc = self._L.efwi_set_model(self._h, C.c_void_p(ts[0].data_ptr()),
                                        C.c_void_p(ts[1].data_ptr()),
                                        C.c_void_p(ts[2].data_ptr()), self._stream())
        check(self._h, rc)

    def set_survey(self, shots: Sequence[Shot], stf) -> None:
        """stf: [nshot, >= nt] source time functions (untapered)."""
        stf = np.ascontiguousarray(np.asarray(stf, dtype=np.float32))
        if stf.ndim != 2 or stf.shape[0] != len(shots) or stf.shape[1] < self.grid.nt:
            raise ValueError(f"stf shape {stf.shape} does not match {len(shots)} shots x nt={self.grid.nt}")
        stf = np.ascontiguousarray(stf[:, :self.grid.nt])
        arr = (EfwiShot * max(len(shots), 1))()
        keep = []
        for k, s in enumerate(shots):
            zr, xr, yr = (np.ascontiguousarray(a, np.int32) for a in (s.z_rec, s.x_rec, s.y_rec))
            keep += [zr, xr, yr]
            e = arr[k]
            e.z_src, e.x_src, e.y_src = (int(v) for v in s.src)
            e.nrec = len(zr)
            e.z_rec = zr.ctypes.data_as(C.POINTER(C.c_int))
            e.x_rec = xr.ctypes.data_as(C.POINTER(C.c_int))
            e.y_rec = yr.ctypes.data_as(C.POINTER(C.c_int))
            for name in ("win_start", "win_end", "weights"):
                v = getattr(s, name)
                if v is not None:
                    v = np.ascontiguousarray(v, np.float32)
                    keep.append(v)
                    setattr(e, name, v.ctypes.data_as(C.POINTER(C.c_float)))
            e.src_weight = float(s.src_weight)
        with torch.cuda.device(self.device):
            rc = self._L.efwi_set_survey(self._h, len(shots), arr,
                                         stf.ctypes.data_as(C.POINTER(C.c_float)))
        check(self._h, rc)
        self.shots = list(shots)

    # ------------------------------------------------------------ utilities
    def trace_sizes(self, shot_ids: Sequence[int]) -> List[int]:
        # Unknown ids count as empty here; the engine rejects them with its
        # own message (after its call-order checks).
        return [3 * self.shots[k].nrec * self.grid.nt if 0 <= k < len(self.shots) else 0
                for k in shot_ids]

    def split(self, flat: torch.Tensor, shot_ids: Sequence[int]) -> List[torch.Tensor]:
        out, off = [], 0
        for k in shot_ids:
            n = 3 * self.shots[k].nrec * self.grid.nt
            out.append(flat[off:off + n].view(3, self.shots[k].nrec, self.grid.nt))
            off += n
        return out

    @staticmethod
    def _ids(shot_ids) -> np.ndarray:
        return np.ascontiguousarray(np.asarray(shot_ids, dtype=np.int32).ravel())

    # ---------------------------------------------------------------- calls
    def forward(self, shot_ids, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Receiver traces of the shots, concatenated [3][nrec][nt] blocks."""
        ids = self._ids(shot_ids)
        n = sum(self.trace_sizes(ids))
        if out is None:
            out = torch.empty(max(n, 1), device=self.device, dtype=torch.float32)[:n]
        with torch.cuda.device(self.device):
            rc = self._L.efwi_forward(self._h, len(ids), ids.ctypes.data_as(C.POINTER(C.c_int)),
                                      C.c_void_p(out.data_ptr()), self._stream())
        check(self._h, rc)
        return out

    def misfit(self, shot_ids, obs: torch.Tensor) -> float:
        ids = self._ids(shot_ids)
        obs = _f32_dev(obs, self.device)
        J = C.c_double(0.0)
        with torch.cuda.device(self.device):
            rc = self._L.efwi_misfit(self._h, len(ids), ids.ctypes.data_as(C.POINTER(C.c_int)),
                                     C.c_void_p(obs.data_ptr()), C.byref(J), self._stream())
        check(self._h, rc)
        return J.value

    def gradient(self, shot_ids, obs: torch.Tensor, mode: str = "reference",
                 want_residual: bool = False, out: Optional[torch.Tensor] = None):
        """Misfit and gradients w.r.t. lambda, mu, rho (device tensors).

        `out`, if given, is a contiguous float32 device tensor of at least
        3 * nz * nx * ny elements: the three images are written into it one
        after the other (and returned as views), so that a caller can sum
        them over ranks with one collective."""
        ids = self._ids(shot_ids)
        obs = _f32_dev(obs, self.device)
        if self.shots and all(0 <= k < len(self.shots) for k in ids) and \
                obs.numel() != sum(self.trace_sizes(ids)):
            raise ValueError("observed data size does not match the shots")
        m = {"reference": _lib.MODE_REFERENCE, "exact": _lib.MODE_EXACT}[mode]
        shp = self.grid.shape
        if out is not None:
            n = self.grid.ncell
            if (out.dtype != torch.float32 or out.device != self.device
                    or not out.is_contiguous() or out.numel() < 3 * n):
                raise ValueError("out must be a contiguous float32 tensor of >= 3 volumes "
                                 "on the engine's device")
            flat = out.view(-1)
            gl, gm, gr = (flat[k * n:(k + 1) * n].view(shp) for k in range(3))
        else:
            gl, gm, gr = (torch.empty(shp, device=self.device, dtype=torch.float32)
                          for _ in range(3))
        res = torch.empty_like(obs) if want_residual else None
        J = C.c_double(0.0)
        with torch.cuda.device(self.device):
            rc = self._L.efwi_gradient(self._h, len(ids), ids.ctypes.data_as(C.POINTER(C.c_int)),
                                       C.c_void_p(obs.data_ptr()), m, C.byref(J),
                                       C.c_void_p(gl.data_ptr()), C.c_void_p(gm.data_ptr()),
                                       C.c_void_p(gr.data_ptr()),
                                       C.c_void_p(res.data_ptr() if res is not None else 0),
                                       self._stream())
        check(self._h, rc)
        if want_residual:
            return J.value, gl, gm, gr, res
        return J.value, gl, gm, gr

    def stf_gradient(self, shot_ids, obs: torch.Tensor):
        """Exact misfit gradient with respect to the (untapered) source-time
        functions of the shots, [n, nt], besides J and the model images."""
        ids = self._ids(shot_ids)
        gs = torch.zeros(len(ids), self.grid.nt, device=self.device, dtype=torch.float32)
        check(self._h, self._L.efwi_set_stf_gradient(self._h, C.c_void_p(gs.data_ptr())))
        try:
            out = self.gradient(shot_ids, obs, mode="exact")
        finally:
            check(self._h, self._L.efwi_set_stf_gradient(self._h, C.c_void_p(0)))
        return out + (gs,)

    def set_scratch(self, syn_w=None, obs_w=None, res=None) -> None:
        """Device buffers (traces layout of the next calls' obs) that every
        misfit also fills with windowed synthetics, windowed observed data
        and the adjoint source; None disables."""
        self._scratch = (syn_w, obs_w, res)
        ptr = [C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)
               for t in (syn_w, obs_w, res)]
        check(self._h, self._L.efwi_set_scratch(self._h, *ptr))

    def forward_windows(self, shot_ids, windows, use_graph: bool = True) -> torch.Tensor:
        """Traces of shots each on its own window (x0, y0, nx, ny) of the
        padded grid: per-window TMA launches on several streams (variant 1)
        or one persistent multi-domain launch per half-step (variant 0)."""
        ids = self._ids(shot_ids)
        if len(windows) != len(ids):
            raise ValueError("one window per shot")
        arr = (_lib.EfwiWindow * max(len(ids), 1))()
        for k, w in enumerate(windows):
            arr[k].x0, arr[k].y0, arr[k].nx, arr[k].ny = (int(v) for v in w)
        out = torch.zeros(sum(self.trace_sizes(ids)), device=self.device, dtype=torch.float32)
        with torch.cuda.device(self.device):
            rc = self._L.efwi_forward_windows(self._h, len(ids), ids.ctypes.data_as(C.POINTER(C.c_int)),
                                              C.cast(arr, C.c_void_p), C.c_void_p(out.data_ptr()),
                                              int(bool(use_graph)), self._stream())
        check(self._h, rc)
        return out

    def gradient_windows(self, shot_ids, windows, obs: torch.Tensor, mode: str = "reference"):
        """Misfit and lambda/mu/rho gradients of shots each on its own window
        (x0, y0, nx, ny) of the padded grid (efwi_gradient_windows): the
        receivers inside a window take part, the images are added into the
        full grid at the window's place."""
        ids = self._ids(shot_ids)
        if len(windows) != len(ids):
            raise ValueError("one window per shot")
        obs = _f32_dev(obs, self.device)
        if obs.numel() != sum(self.trace_sizes(ids)):
            raise ValueError("observed data size does not match the shots")
        arr = (_lib.EfwiWindow * max(len(ids), 1))()
        for k, w in enumerate(windows):
            arr[k].x0, arr[k].y0, arr[k].nx, arr[k].ny = (int(v) for v in w)
        m = {"reference": _lib.MODE_REFERENCE, "exact": _lib.MODE_EXACT}[mode]
        gl, gm, gr = (torch.empty(self.grid.shape, device=self.device, dtype=torch.float32)
                      for _ in range(3))
        J = C.c_double(0.0)
        with torch.cuda.device(self.device):
            rc = self._L.efwi_gradient_windows(
                self._h, len(ids), ids.ctypes.data_as(C.POINTER(C.c_int)), C.cast(arr, C.c_void_p),
                C.c_void_p(obs.data_ptr()), m, C.byref(J), C.c_void_p(gl.data_ptr()),
                C.c_void_p(gm.data_ptr()), C.c_void_p(gr.data_ptr()), self._stream())
        check(self._h, rc)
        return J.value, gl, gm, gr

    def adjoint(self, shot_ids, adj_src: torch.Tensor):
        """J^T adj_src: exact adjoint images (lambda, mu, rho) of the shots
        for an adjoint source in the traces layout."""
        ids = self._ids(shot_ids)
        w = _f32_dev(adj_src, self.device)
        if w.numel() != sum(self.trace_sizes(ids)):
            raise ValueError("adjoint source size does not match the shots")
        shp = self.grid.shape
        gl, gm, gr = (torch.empty(shp, device=self.device, dtype=torch.float32) for _ in range(3))
        with torch.cuda.device(self.device):
            rc = self._L.efwi_adjoint(self._h, len(ids), ids.ctypes.data_as(C.POINTER(C.c_int)),
                                      C.c_void_p(w.data_ptr()), C.c_void_p(gl.data_ptr()),
                                      C.c_void_p(gm.data_ptr()), C.c_void_p(gr.data_ptr()),
                                      self._stream())
        check(self._h, rc)
        return gl, gm, gr

    def illumination(self, shot_ids):
        """Diagonal pseudo-Hessian (source illumination) of lambda, mu, rho."""
        ids = self._ids(shot_ids)
        shp = self.grid.shape
        hl, hm, hr = (torch.empty(shp, device=self.device, dtype=torch.float32) for _ in range(3))
        with torch.cuda.device(self.device):
            rc = self._L.efwi_illumination(self._h, len(ids), ids.ctypes.data_as(C.POINTER(C.c_int)),
                                           C.c_void_p(hl.data_ptr()), C.c_void_p(hm.data_ptr()),
                                           C.c_void_p(hr.data_ptr()), self._stream())
        check(self._h, rc)
        return hl, hm, hr

    # ------------------------------------------------- exact-adjoint support
    def set_checkpoint_budget(self, nbytes: int) -> None:
        """HBM bytes for the exact gradient's checkpoint slots."""
        check(self._h, self._L.efwi_set_checkpoint_budget(self._h, int(nbytes)))

    def state_bytes(self) -> int:
        """Bytes of one checkpointed state (9 fields + C-PML slabs)."""
        return int(self._L.efwi_state_bytes(self._h))

    def checkpoint_stats(self) -> dict:
        fs, sl = C.c_longlong(0), C.c_int(0)
        check(self._h, self._L.efwi_checkpoint_stats(self._h, C.byref(fs), C.byref(sl)))
        return {"forward_steps": fs.value, "slots": sl.value}

    def step(self, state: torch.Tensor, transpose: bool = False) -> torch.Tensor:
        """One source-free forward step (or its exact transpose) of a
        [27, nz, nx, ny] state: 9 fields then 18 C-PML memory variables in
        the oracle's order.  Returns the new state (a device copy)."""
        st = _f32_dev(state, self.device).clone()
        if tuple(st.shape) != (27,) + tuple(self.grid.shape):
            raise ValueError(f"state shape {tuple(st.shape)} != (27, {self.grid.shape})")
        with torch.cuda.device(self.device):
            rc = self._L.efwi_step(self._h, C.c_void_p(st.data_ptr()), int(bool(transpose)),
                                   self._stream())
        check(self._h, rc)
        return st

    # ------------------------------------------------------------ profiling
    def profile(self, sample: int) -> None:
        check(self._h, self._L.efwi_profile(self._h, int(sample)))

    def profile_read(self) -> dict:
        n = self._L.efwi_kernel_count()
        timed = (C.c_longlong * n)()
        ms = (C.c_double * n)()
        launches = (C.c_longlong * n)()
        check(self._h, self._L.efwi_profile_read(self._h, n, timed, ms, launches))
        names = _lib.kernel_names()
        return {names[k]: {"timed": timed[k], "ms": ms[k], "launches": launches[k]}
                for k in range(n)}
