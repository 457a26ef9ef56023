"""A lost step, as Jobs.lost is in the reference (src/core/jobs.js:384-391), made without a fault:
every device wait is bounded by the context's budget (bg_set_wait_budget).  A budget of one
iteration makes the grid's first wait run out; the status word ends every other wait, the call
returns BG_ETIMEOUT with its message, and the same context then solves the same step, bit for bit
as the oracle does, once the budget is back to its default."""
import ctypes as C

import pytest

import oracle_io
from stage_io import StageCopy, first_difference
from bearing_b200 import _ffi, scenes
from bearing_b200.world import World

pytestmark = pytest.mark.gpu

DT = 1 / 60


def test_a_wait_that_runs_out_loses_the_step_and_the_context_goes_on():
    w = World({}, solver=oracle_io.solver(0))
    scenes.pyramid(w)
    for _ in range(3):
        w.step(DT)
    w.begin_step(DT)
    base = StageCopy(w)
    g = _ffi.gpu()
    ctx = g.bg_create(0, _ffi.BG_FLAG_GRID)
    try:
        assert g.bg_set_wait_budget(ctx, 1) == 0
        lost = base.copy()
        B, R, S = lost.views()
        assert g.bg_solve_step(ctx, C.byref(B), C.byref(R), C.byref(S)) == _ffi.BG_ETIMEOUT
        assert "budget" in g.bg_last_error(ctx).decode()
        assert g.bg_set_wait_budget(ctx, 0) == 0
        again = base.copy()
        B, R, S = again.views()
        assert g.bg_solve_step(ctx, C.byref(B), C.byref(R), C.byref(S)) == 0, g.bg_last_error(ctx).decode()
        assert first_difference(oracle_io.solve(base.copy()), again) is None
        assert g.bg_set_wait_budget(ctx, -1) == _ffi.BG_EINVAL
    finally:
        g.bg_destroy(ctx)
