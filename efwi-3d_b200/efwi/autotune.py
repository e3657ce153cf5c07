"""Launch-configuration autotuner of the TMA stencil kernels.

The kernels' results do not depend on the configuration (tile, ring depth,
occupancy target, z planes per CTA); only their speed does.  For one
problem the tuner runs short gradient probes (the time loops stopped after
`nt_probe` steps) on the handle's real grid, model and survey, reads the
per-kernel CUDA-event timings of the engine, and keeps the fastest forward
and reverse configurations.
"""
from __future__ import annotations

import itertools
from typing import Dict, Sequence

import torch

FWD_CFGS = (0, 1, 2, 3)
REV_CFGS = (0, 1, 2, 3, 4, 5, 6, 7)
ZCHUNKS = (2, 3, 4, 6, 8)


def _probe(P, shot_ids, obs, names) -> float:
    P.profile(1)
    P.profile_read()
    P.gradient(shot_ids, obs)
    torch.cuda.synchronize(P.device)
    prof = P.profile_read()
    t = 0.0
    for n in names:
        v = prof.get(n, {})
        if not v.get("timed"):
            return float("inf")
        t += v["ms"] / v["timed"]
    return t


def _time_call(P, ids, obs, reps: int = 2) -> float:
    """Fastest of `reps` reference-mode gradient calls (ms, CUDA events on
    the current stream; the call is synchronous, its lanes included)."""
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        P.gradient(ids, obs)
        e1.record()
        torch.cuda.synchronize(P.device)
        best = min(best, e0.elapsed_time(e1))
    return best


def autotune(P, shot_id: int, obs_shot: torch.Tensor, nt_probe: int = 16,
             fwd_cfgs: Sequence[int] = FWD_CFGS, rev_cfgs: Sequence[int] = REV_CFGS,
             zchunks: Sequence[int] = ZCHUNKS, pair_ids=None, pair_obs=None,
             lanes_nt: int = 160, lanes_reps: int = 3) -> Dict:
    """Tunes `P` (a Propagator with model and survey set) on shot `shot_id`
    whose observed traces are `obs_shot`; returns the timings and the choice.

    With two shots `pair_ids` (observed traces `pair_obs`) and more than
    one lane on P, a last stage times whole two-shot calls, whose lanes
    share the GPU, for the chosen z planes per CTA and 8 (forward and
    reverse): concurrent lanes fill each other's tail waves, which favours
    longer z marches than the kernels timed alone do.  Those candidates
    differ by a few per cent, so each is timed `lanes_reps` times over
    `lanes_nt` steps and its fastest run counts."""
    ids = [int(shot_id)]
    P.set_nt_limit(nt_probe)
    try:
        cur = getattr(P, "tuning", (0, 8, 0, 8))
        fwd = {}
        for cfg, zc in itertools.product(fwd_cfgs, zchunks):
            P.set_tuning(cfg, zc, cur[2], cur[3])
            _probe(P, ids, obs_shot, ())  # warm (first launch sets attributes)
            fwd[(cfg, zc)] = _probe(P, ids, obs_shot, ("stress_fwd", "velocity_fwd"))
        bf = min(fwd, key=fwd.get)
        rev = {}
        for cfg, zc in itertools.product(rev_cfgs, zchunks):
            P.set_tuning(bf[0], bf[1], cfg, zc)
            _probe(P, ids, obs_shot, ())
            rev[(cfg, zc)] = _probe(P, ids, obs_shot, ("rev_velocity", "rev_stress"))
        br = min(rev, key=rev.get)
    finally:
        P.set_nt_limit(0)
        P.profile(0)
    zf, zr = bf[1], br[1]
    pair = {}
    if pair_ids is not None and len(pair_ids) >= 2 and getattr(P, "lanes", 1) > 1:
        P.set_nt_limit(lanes_nt)
        try:
            for cand in sorted({(zf, zr), (8, zr), (zf, 8), (8, 8)}):
                P.set_tuning(bf[0], cand[0], br[0], cand[1])
                _time_call(P, pair_ids, pair_obs, reps=1)  # warm
                pair[cand] = _time_call(P, pair_ids, pair_obs, reps=lanes_reps)
        finally:
            P.set_nt_limit(0)
        zf, zr = min(pair, key=pair.get)
    P.set_tuning(bf[0], zf, br[0], zr)
    out = {"fwd_cfg": bf[0], "zchunk_fwd": zf, "rev_cfg": br[0], "zchunk_rev": zr,
           "fwd_ms": round(fwd[bf], 4), "rev_ms": round(rev[br], 4),
           "fwd_default_ms": round(fwd.get((0, 8), float("nan")), 4),
           "rev_default_ms": round(rev.get((0, 8), float("nan")), 4),
           "probes": len(fwd) + len(rev) + len(pair)}
    if pair:
        out["lanes_probe_ms"] = {f"{a},{b}": round(v, 3) for (a, b), v in pair.items()}
    return out


def autotune_windows(P, shot_ids, windows, nt_probe: int = 16, bxs=(4, 8), zchunks=(4, 8, 16),
                     fwd_cfgs: Sequence[int] = FWD_CFGS, tma_zchunks=(2, 4, 8)):
    """Stencil variant and launch shape of the window forward, the fastest
    over short probes (time loop stopped after `nt_probe` steps, CUDA events
    on the current stream): the L1-served multi-domain launch over
    (tile_bx, zchunk) and the per-window TMA kernels over (fwd_cfg, zchunk).
    Sets the choice on P (its variant included: the windows' results do not
    depend on it)."""
    def probe():
        P.forward_windows(shot_ids, windows, use_graph=True)  # warm
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        P.forward_windows(shot_ids, windows, use_graph=True)
        e1.record()
        torch.cuda.synchronize(P.device)
        return e0.elapsed_time(e1)

    cur = getattr(P, "tuning", (0, 8, 0, 8))
    P.set_nt_limit(nt_probe)
    times = {}
    try:
        P.set_variant(0)
        for bx, zc in itertools.product(bxs, zchunks):
            P.set_options(if_win=P.if_win, tile_bx=bx, zchunk=zc)
            times[("l1", bx, zc)] = probe()
        P.set_variant(1)
        for cfg, zc in itertools.product(fwd_cfgs, tma_zchunks):
            P.set_tuning(cfg, zc, cur[2], cur[3])
            times[("tma", cfg, zc)] = probe()
    finally:
        P.set_nt_limit(0)
    best = min(times, key=times.get)
    if best[0] == "l1":
        P.set_variant(0)
        P.set_options(if_win=P.if_win, tile_bx=best[1], zchunk=best[2])
        out = {"variant": "l1", "tile_bx": best[1], "zchunk": best[2]}
    else:
        P.set_variant(1)
        P.set_tuning(best[1], best[2], cur[2], cur[3])
        out = {"variant": "tma", "fwd_cfg": best[1], "zchunk": best[2]}
    best_l1 = min(v for k, v in times.items() if k[0] == "l1")
    best_tma = min(v for k, v in times.items() if k[0] == "tma")
    out.update({"probe_ms": round(times[best], 3), "best_l1_ms": round(best_l1, 3),
                "best_tma_ms": round(best_tma, 3), "probes": len(times)})
    return out
