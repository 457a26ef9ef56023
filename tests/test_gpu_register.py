"""bg_register_host: the caller's own columns page-locked in place, so that bg_solve_step copies
them directly.  Results never depend on it, and the written columns only slipped() reads after
the stage (sliding, anchor_a, anchor_b) may be left NULL, in which case nothing is copied back
into them and every other column is the same."""
import ctypes as C

import numpy as np
import pytest

import oracle_io
from stage_io import StageCopy, first_difference
from bearing_b200 import _ffi, scenes
from bearing_b200.world import World

pytestmark = pytest.mark.gpu

DT = 1 / 60


def pile_input(steps=60):
    w = World({}, solver=oracle_io.solver(0))
    scenes.pile(w, count=400, seed=3, extent=8.0)
    for _ in range(steps):
        w.step(DT)
    w.begin_step(DT)
    return StageCopy(w)


def solve(lib, ctx, copy, trim=False):
    B, R, S = copy.views()
    if trim:
        R.sliding = None
        R.anchor_a = None
        R.anchor_b = None
    rc = lib.bg_solve_step(ctx, C.byref(B), C.byref(R), C.byref(S))
    assert rc == 0, lib.bg_last_error(ctx)
    return copy


def test_registered_columns_give_the_same_step():
    base = pile_input()
    assert base.solved > 100
    want = oracle_io.solve(base.copy())
    lib = _ffi.gpu()
    ctx = lib.bg_create(0, 0)
    try:
        work = base.copy()
        B, R, _ = work.views()
        assert lib.bg_registered_bytes(ctx) == 0
        assert lib.bg_register_host(ctx, C.byref(B), C.byref(R), work.count) == 0, lib.bg_last_error(ctx)
        held = lib.bg_registered_bytes(ctx)
        payload = sum(v.nbytes for v in work.body.values()) + sum(v.nbytes for v in work.rows.values())
        assert held >= payload, (held, payload)
        for _ in range(3):   # the same arrays, refilled, as a World steps
            work.fill(base)
            got = solve(lib, ctx, work)
            assert first_difference(want, got) is None, first_difference(want, got)
        # registering again replaces what was held (a World whose columns grew)
        bigger = base.copy()
        B2, R2, _ = bigger.views()
        assert lib.bg_register_host(ctx, C.byref(B2), C.byref(R2), bigger.count) == 0
        got = solve(lib, ctx, bigger)
        assert first_difference(want, got) is None
        assert lib.bg_unregister_host(ctx) == 0
        assert lib.bg_registered_bytes(ctx) == 0
        # and the arrays work as ordinary memory again
        again = solve(lib, ctx, base.copy())
        assert first_difference(want, again) is None
    finally:
        lib.bg_destroy(ctx)


def test_a_row_capacity_short_of_the_rows_is_refused():
    base = pile_input(10)
    lib = _ffi.gpu()
    ctx = lib.bg_create(0, 0)
    try:
        B, R, _ = base.views()
        assert lib.bg_register_host(ctx, C.byref(B), C.byref(R), base.count - 1) == _ffi.BG_EINVAL
        assert lib.bg_registered_bytes(ctx) == 0
    finally:
        lib.bg_destroy(ctx)


def test_columns_registered_short_of_a_call_are_staged():
    # Registered for fewer rows than a later call moves: those columns go through the staging
    # block (a copy past a registered range would read unlocked pages), with the same results.
    base = pile_input()
    want = oracle_io.solve(base.copy())
    lib = _ffi.gpu()
    ctx = lib.bg_create(0, 0)
    try:
        work = base.copy()
        B, R, _ = work.views()
        R.count = work.count // 2
        assert lib.bg_register_host(ctx, C.byref(B), C.byref(R), R.count) == 0
        got = solve(lib, ctx, work)
        assert first_difference(want, got) is None
    finally:
        lib.bg_destroy(ctx)


def test_slipped_only_outputs_may_be_null():
    base = pile_input()
    want = oracle_io.solve(base.copy())
    lib = _ffi.gpu()
    ctx = lib.bg_create(0, 0)
    try:
        work = base.copy()
        before = {f: work.rows[f].copy() for f in ("sliding", "anchor_a", "anchor_b")}
        got = solve(lib, ctx, work, trim=True)
        for f, v in before.items():
            assert np.array_equal(got.rows[f], v), f"{f} was written"   # no array was passed for it
            got.rows[f][:] = want.rows[f]
        assert first_difference(want, got) is None, first_difference(want, got)
    finally:
        lib.bg_destroy(ctx)
