"""Binomial checkpointing schedule (cfdb_revolve_plan), host only: the
schedule reverses every step in order from the right state, never uses more
slots than given, and performs the optimal number of forward steps
r*l - C(s+r, s+1) for the smallest r with C(s+r, s) >= l (Griewank and
Walther, ACM TOMS 26(1) 2000)."""
from __future__ import annotations

from math import comb

import pytest


def simulate(plan, steps, snaps):
    RV_ADVANCE, RV_TAKESHOT, RV_RESTORE, RV_FIRSTURN, RV_YOUTURN = 1, 2, 3, 4, 5
    slots = {}
    cur = 0
    turns = []
    fwd = 0
    for act, arg, at in plan:
        if act == RV_TAKESHOT:
            assert 0 <= arg < snaps
            slots[arg] = cur
            assert at == cur
        elif act == RV_RESTORE:
            assert arg in slots and slots[arg] == at
            cur = slots[arg]
        elif act == RV_ADVANCE:
            assert at == cur and arg > 0
            cur += arg
            fwd += arg
        elif act in (RV_FIRSTURN, RV_YOUTURN):
            assert at == cur, (at, cur)
            assert (act == RV_FIRSTURN) == (len(turns) == 0)
            turns.append(at)
            cur = None
        else:
            raise AssertionError(act)
    assert turns == list(range(steps - 1, -1, -1))
    return fwd


def optimal_forward(l, s):
    if s >= l:
        return l - 1
    r = 0
    while comb(s + r, s) < l:
        r += 1
    return r * l - comb(s + r, s + 1)


@pytest.mark.parametrize("steps", [1, 2, 3, 7, 10, 25, 64, 100, 400])
@pytest.mark.parametrize("snaps", [1, 2, 3, 5, 8, 27, 400])
def test_schedule_valid_and_optimal(cfdb, steps, snaps):
    plan, fwd = cfdb.revolve_plan(steps, snaps)
    got = simulate(plan, steps, min(snaps, steps))
    assert got == fwd
    assert fwd == optimal_forward(steps, min(snaps, steps))


def test_plan_rejects_bad_arguments(cfdb):
    import ctypes as C
    cnt = C.c_int64()
    L = cfdb.lib()
    assert L.cfdb_revolve_plan(0, 3, None, None, None, 0, C.byref(cnt), None) == cfdb.capi.EINVAL
    assert L.cfdb_revolve_plan(5, 0, None, None, None, 0, C.byref(cnt), None) == cfdb.capi.EINVAL
