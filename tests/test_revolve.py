"""Binomial checkpoint schedule of the exact gradient (host code of the C
ABI, no GPU): every adjoint block sees its own state, the first sweep is
uninterrupted, the slot count is respected, and the number of forward steps
is the published minimum t*l - C(s+t+1, t-1) (Griewank & Walther 2000)."""
from math import comb

import pytest

from efwi import _lib

ADVANCE, STORE, RESTORE, BLOCK = 0, 1, 2, 3


def _simulate(nt, slots, actions):
    """Replays a schedule on state indices; returns blocks in run order,
    forward steps, the state index of the first block and whether the
    first sweep was uninterrupted."""
    cur = 0
    store = {}
    blocks, steps = [], 0
    first_sweep_clean = True
    for op, a, b in actions:
        if op == ADVANCE:
            assert cur == a, (cur, a)
            assert b > a
            steps += b - a
            cur = b
        elif op == STORE:
            assert 0 <= a < slots
            store[a] = cur
        elif op == RESTORE:
            if not blocks:
                first_sweep_clean = False
            cur = 0 if a < 0 else store[a]
        else:
            assert cur == a, ("block", a, "sees state", cur)
            blocks.append(a)
    return blocks, steps, first_sweep_clean


def _tmin(nt, s):
    t = 1
    while comb(s + t + 1, t) < nt:
        t += 1
    return t


@pytest.mark.parametrize("nt,slots", [(2, 1), (7, 1), (10, 2), (57, 3), (80, 2), (100, 5),
                                      (300, 8), (1000, 20), (4000, 46), (64, 63), (64, 200)])
def test_schedule_is_valid_and_optimal(nt, slots):
    info = _lib.checkpoint_plan(nt, slots, with_actions=True)
    blocks, steps, clean = _simulate(nt, slots, info["actions"])
    assert blocks == list(range(nt - 1, -1, -1))
    assert clean
    assert steps == info["forward_steps"]
    assert info["slots_used"] <= slots
    s = min(slots, nt - 1)
    t = _tmin(nt, s)
    assert info["repetitions"] == t
    assert steps == t * nt - comb(s + t + 1, t - 1)


def test_storing_every_state_advances_each_step_once():
    info = _lib.checkpoint_plan(500, 499)
    assert info["forward_steps"] == 499 and info["repetitions"] == 1


def test_no_slots_recomputes_from_the_start():
    nt = 30
    info = _lib.checkpoint_plan(nt, 0, with_actions=True)
    blocks, steps, clean = _simulate(nt, 0, info["actions"])
    assert blocks == list(range(nt - 1, -1, -1)) and clean
    assert steps == nt * (nt - 1) // 2


def test_config3_budget_schedule():
    """Config 3 (120^3 padded, nt 4000) under 4 GiB: 9 fields + C-PML slabs
    per state (np 12), about 87 MB, so 49 slots and 3 repetitions."""
    n, np_ = 120, 12
    state = 4 * (9 * n * n * n + 6 * 3 * 2 * np_ * n * n)
    slots = (4 << 30) // state
    info = _lib.checkpoint_plan(4000, slots)
    assert slots == 49
    assert info["repetitions"] == 3
    assert info["forward_steps"] < 3 * 4000
