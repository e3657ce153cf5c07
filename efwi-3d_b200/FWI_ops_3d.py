"""Drop-in for the reference's Ops/FWI/FWI_ops_3d.py.

Exposes the same objects with the same signatures and return values:

* ``fwi_ops.forward(Lambda, Mu, Den, stf, gpu_id, shot_ids, para_fname)``
  -> ``[misfit]``                                    (Torch_Fwi.cpp:12-31)
* ``fwi_ops.backward(Lambda, Mu, Den, stf, ngpu, shot_ids, para_fname)``
  -> ``[misfit, grad_Lambda, grad_Mu, grad_Den, grad_stf]`` (Torch_Fwi.cpp:33-97)
* ``fwi_ops.obscalc(...)`` writes ``Shot_{x,y,z}{id}.bin`` (Torch_Fwi.cpp:99-125)
* ``FWIFunction``, ``FWI_3d``, ``FWI_obscalc``         (FWI_ops_3d.py:34-108)

Underneath, calls go to the B200 engine (libefwi.so) through
:mod:`efwi.engine`.  Model tensors may live on the CPU (as in the
reference's drivers) or on a GPU; results come back on the input's device.
The engine keeps the grid, survey, workspace and observed data resident in
HBM between calls of the same para file.  Errors raise exceptions instead of
ending the process.
"""
from __future__ import annotations

import os
import threading
from typing import Dict, List, Optional, Tuple

import numpy as np
import torch
import torch.nn as nn

import fwi_utils as ft
from efwi import config as _cfg
from efwi.autotune import autotune
from efwi.engine import Propagator

__all__ = ["fwi_ops", "FWIFunction", "FWI_3d", "FWI_obscalc", "set_lanes", "set_tuning"]


def _mtime(path: str) -> Tuple[float, int]:
    st = os.stat(path)
    return (st.st_mtime, st.st_size)


# Shots of one gradient call that run concurrently on a GPU, each lane with
# its own workspace and stream (the reference runs them one after another,
# libCUFD.cu:220-798).  A lane beyond the first holds its own state (about
# 21 volumes) and boundary-shell store (9 floats per shell point and time
# step: 37.6 GB at 152^3 and nt 2000) outside torch's allocator.  Set with
# set_lanes(n) or FWI_3d(..., opt={"lanes": n}); a lane that does not fit in
# device memory at the call is left out.
LANES = 2
_lanes_by_para: Dict[str, int] = {}


# Launch configuration of later sessions: None autotunes on a session's
# first gradient call; a tuple (fwd_cfg, zchunk_fwd, rev_cfg, zchunk_rev)
# is used as it is (efwi_set_tuning).
TUNING: Optional[Tuple[int, int, int, int]] = None


def set_tuning(tuning: Optional[Tuple[int, int, int, int]]) -> None:
    """Fixes the stencil launch configuration of the sessions (None: the
    autotuner picks it on a session's first gradient call)."""
    global TUNING
    TUNING = None if tuning is None else tuple(int(v) for v in tuning)
    for s in _sessions.values():
        s.tuned = False


def set_lanes(n: int, para_fname: Optional[str] = None) -> None:
    """Concurrent shots of later gradient calls: for every para file, or
    (para_fname given) for that one."""
    n = int(n)
    if not 1 <= n <= 8:
        raise ValueError("lanes must be in [1, 8]")
    global LANES
    if para_fname is None:
        LANES = n
    else:
        _lanes_by_para[os.path.abspath(para_fname)] = n


class _Session:
    """Engine state of one para file on one device."""

    def __init__(self, para_fname: str, device: torch.device):
        self.para_fname = para_fname
        self.device = device
        self.prop: Optional[Propagator] = None
        self.para_key = None
        self.survey_key = None
        self.stf_cache: Optional[np.ndarray] = None
        self.obs_cache: Dict[int, Tuple[tuple, torch.Tensor]] = {}
        self.lock = threading.Lock()
        self.tuned = False

    def refresh(self, stf: torch.Tensor) -> "_cfg.Para":
        pk = _mtime(self.para_fname)
        if pk != self.para_key or self.prop is None:
            self.para = _cfg.read_para(self.para_fname)
            g = self.para.grid
            if self.prop is None or (self.prop.grid != g):
                if self.prop is not None:
                    self.prop.close()
                self.prop = Propagator(g, device=self.device, if_win=self.para.if_win)
                self.survey_key = None
                self.stf_cache = None
                self.tuned = False
            else:
                self.prop.set_options(if_win=self.para.if_win)
            self.para_key = pk
        self.prop.set_lanes(_lanes_by_para.get(self.para_fname, LANES))
        sk = (self.para.survey_fname, _mtime(self.para.survey_fname))
        stf_np = stf.detach().to("cpu", torch.float32).contiguous().numpy()
        if sk != self.survey_key or self.stf_cache is None or not np.array_equal(stf_np, self.stf_cache):
            self.shots = _cfg.read_survey(self.para.survey_fname, self.para.grid.npml,
                                          self.para.if_win)
            nt = self.para.grid.nt
            flat = stf_np.reshape(-1)
            rows = np.zeros((len(self.shots), nt), np.float32)
            for k in range(len(self.shots)):
                # stf(shot_id, it) = stf[shot_id * nSteps + it] (Src_Rec.cu:9,140-142)
                if (k + 1) * nt <= flat.size:
                    rows[k] = flat[k * nt:(k + 1) * nt]
            self.nstf_rows = flat.size // nt
            present = [s if s is not None else _cfg.Shot(src=(2, 2, 2), z_rec=np.zeros(0, int),
                                                          x_rec=np.zeros(0, int),
                                                          y_rec=np.zeros(0, int))
                       for s in self.shots]
            self.prop.set_survey(present, rows)
            self.survey_key = sk
            self.stf_cache = stf_np.copy()
        return self.para

    def check_ids(self, ids: List[int]) -> None:
        for k in ids:
            if k < 0 or k >= len(self.shots) or self.shots[k] is None:
                raise ValueError(f"shot {k} is not in the survey {self.para.survey_fname}")
            if k >= self.nstf_rows:
                raise ValueError(f"stf has no row for shot {k}")

    def observed(self, ids: List[int]) -> torch.Tensor:
        """Observed data of the shots, concatenated [3][nrec][nt] blocks,
        cached in HBM while the files are unchanged."""
        nt = self.para.grid.nt
        parts = []
        for k in ids:
            fn = [_cfg.shot_file(self.para.data_dir_name, c, k) for c in "xyz"]
            key = tuple(_mtime(f) if os.path.exists(f) else None for f in fn)
            hit = self.obs_cache.get(k)
            if hit is None or hit[0] != key:
                arr = _cfg.read_shot_data(self.para.data_dir_name, k, self.shots[k].nrec, nt)
                t = torch.from_numpy(arr.reshape(-1)).to(self.device, non_blocking=False)
                self.obs_cache[k] = (key, t)
                hit = self.obs_cache[k]
            parts.append(hit[1])
        return torch.cat(parts) if parts else torch.zeros(0, device=self.device)


_sessions: Dict[Tuple[str, int], _Session] = {}
_sessions_lock = threading.Lock()


def _session(para_fname: str, device_index: int) -> _Session:
    key = (os.path.abspath(para_fname), device_index)
    with _sessions_lock:
        s = _sessions.get(key)
        if s is None:
            s = _Session(os.path.abspath(para_fname), torch.device("cuda", device_index))
            _sessions[key] = s
    return s


def _shards(ids: List[int], ngpu: int) -> List[List[int]]:
    """Torch_Fwi.cpp:53-54,74-76: bars = linspace(0, n, ngpu+1) cast to int."""
    n = len(ids)
    bars = torch.linspace(0, n, ngpu + 1, dtype=torch.float32)
    cut = [int(b.item()) for b in bars]
    return [ids[cut[i]:cut[i + 1]] for i in range(ngpu)]


def _reduce_shards(results, dev):
    """Sum of the per-GPU (misfit, gλ, gμ, gρ) of the shards in shard order
    (Torch_Fwi.cpp:89-94 adds them on the host).  The images are summed on
    the first shard's device, each other shard's three volumes arriving in
    one peer copy, and the sum then moves to `dev` once; the misfit is
    summed in float32 as the reference's host loop does."""
    J = np.float32(0.0)
    for r in results:
        J += np.float32(r[0])
    base = results[0][1].device
    n = results[0][1].numel()
    shape = results[0][1].shape
    acc = torch.empty(3 * n, dtype=torch.float32, device=base)
    for k in range(3):
        acc[k * n:(k + 1) * n].copy_(results[0][1 + k].reshape(-1))
    if len(results) > 1:
        part = torch.empty_like(acc)
        for r in results[1:]:
            for k in range(3):
                part[k * n:(k + 1) * n].copy_(r[1 + k].reshape(-1), non_blocking=True)
            acc += part
    out = acc.to(dev)
    return float(J), *(out[k * n:(k + 1) * n].view(shape) for k in range(3))


class _scratch:
    """scratch_dir_name (Parameter.cpp:118-124): after the misfit, writes
    Residual_Shot_{x,y,z}{id}.bin, Syn_Shot_... and CondObs_Shot_... --
    the adjoint source, the windowed synthetics and the windowed observed
    data, [nrec][nt] float32 per component (libCUFD.cu:660-700)."""

    def __init__(self, s, ids, obs):
        self.s, self.ids, self.obs = s, ids, obs
        self.on = bool(s.para.scratch_dir_name)

    def __enter__(self):
        if self.on:
            self.bufs = [torch.empty_like(self.obs) for _ in range(3)]
            self.s.prop.set_scratch(*self.bufs)
        return self

    def __exit__(self, et, ev, tb):
        if not self.on:
            return False
        self.s.prop.set_scratch()
        if et is not None:
            return False
        d = self.s.para.scratch_dir_name
        os.makedirs(d, exist_ok=True)
        syn, cobs, res = (self.s.prop.split(b.cpu(), self.ids) for b in self.bufs)
        for k, sid in enumerate(self.ids):
            for c, name in enumerate("xyz"):
                for prefix, arr in (("Residual", res), ("Syn", syn), ("CondObs", cobs)):
                    arr[k][c].numpy().astype(np.float32).tofile(
                        os.path.join(d, f"{prefix}_Shot_{name}{sid}.bin"))
        return False


def _ids_list(shot_ids) -> List[int]:
    return [int(v) for v in torch.as_tensor(shot_ids).reshape(-1).tolist()]


class _FwiOps:
    """The three entry points of the reference extension module."""

    def forward(self, Lambda, Mu, Den, stf, gpu_id, shot_ids, para_fname):
        ids = _ids_list(shot_ids)
        s = _session(para_fname, int(gpu_id))
        with s.lock:
            s.refresh(stf)
            s.check_ids(ids)
            s.prop.set_model(Lambda, Mu, Den)
            obs = s.observed(ids)
            with _scratch(s, ids, obs):
                J = s.prop.misfit(ids, obs)
        return [torch.tensor([J], dtype=torch.float32)]

    def backward(self, Lambda, Mu, Den, stf, ngpu, shot_ids, para_fname):
        ids = _ids_list(shot_ids)
        ngpu = int(ngpu)
        if ngpu < 1 or ngpu > len(ids):
            raise ValueError("The number of GPUs should be smaller than the number of shots!")
        shards = _shards(ids, ngpu)
        results = [None] * ngpu
        errors = [None] * ngpu

        def run(i):
            try:
                s = _session(para_fname, i)
                with s.lock, torch.cuda.device(i):
                    s.refresh(stf)
                    s.check_ids(shards[i])
                    s.prop.set_model(Lambda, Mu, Den)
                    obs = s.observed(shards[i])
                    if not s.tuned and TUNING is not None:
                        s.prop.set_tuning(*TUNING)
                        s.tuned = True
                    if not s.tuned:
                        # launch shapes timed once per session on the real grid
                        nt = s.para.grid.nt
                        n0 = 3 * s.shots[shards[i][0]].nrec * nt
                        two = shards[i][:2] if len(shards[i]) >= 2 else None
                        n1 = n0 + 3 * s.shots[two[1]].nrec * nt if two else 0
                        autotune(s.prop, shards[i][0], obs[:n0], pair_ids=two,
                                 pair_obs=obs[:n1] if two else None)
                        s.tuned = True
                    with _scratch(s, shards[i], obs):
                        results[i] = s.prop.gradient(shards[i], obs)
                    torch.cuda.current_stream(i).synchronize()
            except BaseException as e:  # re-raised on the caller's thread
                errors[i] = e

        if ngpu == 1:
            run(0)
        else:
            th = [threading.Thread(target=run, args=(i,)) for i in range(ngpu)]
            for t in th:
                t.start()
            for t in th:
                t.join()
        for e in errors:
            if e is not None:
                raise e
        dev = Lambda.device if isinstance(Lambda, torch.Tensor) else torch.device("cpu")
        J, gl, gm, gr = _reduce_shards(results, dev)
        gstf = torch.zeros(torch.as_tensor(stf).shape, dtype=torch.float32, device=dev)
        return [torch.tensor([J], dtype=torch.float32), gl, gm, gr, gstf]

    def obscalc(self, Lambda, Mu, Den, stf, ngpu, shot_ids, para_fname):
        ids = _ids_list(shot_ids)
        ngpu = int(ngpu)
        if ngpu < 1 or ngpu > len(ids):
            raise ValueError("The number of GPUs should be smaller than the number of shots!")
        shards = _shards(ids, ngpu)
        errors = [None] * ngpu

        def run(i):
            try:
                s = _session(para_fname, i)
                with s.lock, torch.cuda.device(i):
                    s.refresh(stf)
                    s.check_ids(shards[i])
                    s.prop.set_model(Lambda, Mu, Den)
                    tr = s.prop.forward(shards[i]).cpu()
                    for k, t in zip(shards[i], s.prop.split(tr, shards[i])):
                        _cfg.write_shot_data(s.para.data_dir_name, k, t.numpy())
            except BaseException as e:
                errors[i] = e

        if ngpu == 1:
            run(0)
        else:
            th = [threading.Thread(target=run, args=(i,)) for i in range(ngpu)]
            for t in th:
                t.start()
            for t in th:
                t.join()
        for e in errors:
            if e is not None:
                raise e
        return None


fwi_ops = _FwiOps()


class FWIFunction(torch.autograd.Function):
    """Runs the whole gradient in forward (as the reference does) and returns
    the cached gradients in backward; the incoming grad_misfit is not used
    (FWI_ops_3d.py:34-44)."""

    @staticmethod
    def forward(ctx, Lambda, Mu, Rho, Stf, ngpu, Shot_ids, para_fname):
        outputs = fwi_ops.backward(Lambda, Mu, Rho, Stf, ngpu, Shot_ids, para_fname)
        ctx.outputs = outputs[1:]
        return outputs[0]

    @staticmethod
    def backward(ctx, grad_misfit):
        grad_Lambda, grad_Mu, grad_Rho, grad_stf = ctx.outputs
        return grad_Lambda, grad_Mu, grad_Rho, grad_stf, None, None, None


class FWI_3d(torch.nn.Module):
    """vp, vs, rho (model grid) -> misfit with gradients through autograd
    (FWI_ops_3d.py:47-94).  rho is divided by 1e3 before lambda and mu are
    formed, as in the reference."""

    def __init__(self, Vp, Vs, Rho, Stf, opt, Mask=None):
        super().__init__()
        self.nz = opt['nz']
        self.nx = opt['nx']
        self.ny = opt['ny']
        self.nPml = opt['nPml']
        self.Bounds = {}
        Vp_pad, Vs_pad, Rho_pad = ft.padding_3d(Vp, Vs, Rho, self.nz, self.nx, self.ny, self.nPml)
        self.register_buffer('Vp_ref', Vp_pad.clone().detach())
        self.register_buffer('Vs_ref', Vs_pad.clone().detach())
        self.register_buffer('Rho_ref', Rho_pad.clone().detach())
        self.Vp = nn.Parameter(Vp) if Vp.requires_grad else Vp
        self.Vs = nn.Parameter(Vs) if Vs.requires_grad else Vs
        self.Rho = nn.Parameter(Rho) if Rho.requires_grad else Rho
        if Mask is None:
            # The reference builds a 2-D ones mask that only broadcasts on
            # cubic grids; a full-size ones mask is the same blend.
            self.Mask = torch.ones(tuple(Vp_pad.shape), dtype=torch.float32)
        else:
            self.Mask = Mask
        self.Stf = Stf
        self.para_fname = opt['para_fname']
        if 'lanes' in opt:
            set_lanes(opt['lanes'], self.para_fname)

    def forward(self, Shot_ids, ngpu=1):
        Vp_pad, Vs_pad, Rho_pad = ft.padding_3d(self.Vp, self.Vs, self.Rho, self.nz, self.nx,
                                                self.ny, self.nPml)
        Vp_mask_pad = self.Mask * Vp_pad + (1.0 - self.Mask) * self.Vp_ref
        Vs_mask_pad = self.Mask * Vs_pad + (1.0 - self.Mask) * self.Vs_ref
        Rho_mask_pad = self.Mask * Rho_pad + (1.0 - self.Mask) * self.Rho_ref
        Rho = Rho_mask_pad / 1e3
        Lambda = (Vp_mask_pad ** 2 - 2.0 * Vs_mask_pad ** 2) * Rho
        Mu = Vs_mask_pad ** 2 * Rho
        return FWIFunction.apply(Lambda, Mu, Rho, self.Stf, ngpu, Shot_ids, self.para_fname)


class FWI_obscalc(torch.nn.Module):
    """Synthetic observed data (FWI_ops_3d.py:96-108); rho is used as given."""

    def __init__(self, Vp, Vs, Rho, Stf, opt):
        super().__init__()
        Vp_pad, Vs_pad, Rho_pad = ft.padding_3d(Vp, Vs, Rho, opt['nz'], opt['nx'], opt['ny'],
                                                opt['nPml'])
        self.Lambda = (Vp_pad ** 2 - 2.0 * Vs_pad ** 2) * Rho_pad
        self.Mu = Vs_pad ** 2 * Rho_pad
        self.Rho = Rho_pad
        self.Stf = Stf
        self.para_fname = opt['para_fname']

    def forward(self, Shot_ids, ngpu=1):
        fwi_ops.obscalc(self.Lambda, self.Mu, self.Rho, self.Stf, ngpu, Shot_ids, self.para_fname)
