"""bg_solve_step_static, the entry point that allocates nothing, against the oracle.

It is for callers that cannot allocate device memory themselves: a host runtime that owns every
device buffer in a pool of its own and passes this library only pointers into it, or a per-frame
loop that must not take a cudaMalloc's synchronisation.  Such a caller passes device arrays;
here torch stands in for the caller's pool.  The result must be bit-identical to the oracle's on
the same input, on two calls in a row (the second sees the first's leftovers in the library's
fixed working array, which it must not depend on), on a small world and on one at the limits
(512 slots, ~1,850 rows); and a refused input (colour starts that decrease, an index out of
range) must come back BG_EINVAL with the caller's arrays untouched.  Named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_io
from stage_io import BODY_COLUMNS, ROW_COLUMNS, StageCopy, first_difference
from bearing_b200 import _ffi, scenes
from bearing_b200.world import World

pytestmark = pytest.mark.gpu

DT = 1 / 60
_CT = {np.float64: C.c_double, np.uint8: C.c_uint8, np.int32: C.c_int32}


def solve_static(copy, expect=None):
    """Runs `copy` through bg_solve_step_static with every array in device memory; returns the
    arrays as the call left them.  `expect` is the return code wanted (BG_OK by default)."""
    import torch
    dev = {}

    def put(name, arr):
        t = torch.from_numpy(np.ascontiguousarray(arr)).cuda()
        dev[name] = t
        return t

    B = _ffi.Bodies()
    B.capacity = copy.capacity
    B.awake_count = copy.awake_count
    B.awake_list = C.cast(C.c_void_p(put("awake_list", copy.awake_list).data_ptr()), C.POINTER(C.c_int32))
    for f, dt, _ in BODY_COLUMNS:
        setattr(B, f, C.cast(C.c_void_p(put("b." + f, copy.body[f]).data_ptr()), C.POINTER(_CT[dt])))
    R = _ffi.Rows()
    R.count = copy.count
    R.solved = copy.solved
    R.starts = (C.c_int32 * _ffi.BG_STARTS)(*[int(x) for x in copy.starts])
    for f, dt, _ in ROW_COLUMNS:
        setattr(R, f, C.cast(C.c_void_p(put("r." + f, copy.rows[f]).data_ptr()), C.POINTER(_CT[dt])))
    S = _ffi.Step(copy.dt, copy.substeps, (C.c_double * 3)(*copy.gravity))
    torch.cuda.synchronize()
    rc = _ffi.gpu().bg_solve_step_static(C.byref(B), C.byref(R), C.byref(S), None)
    want = _ffi.BG_OK if expect is None else expect
    assert rc == want, f"bg_solve_step_static returned {rc}, wanted {want}"
    torch.cuda.synchronize()
    out = copy.copy()
    for f, _dt, _ in BODY_COLUMNS:
        out.body[f][:] = dev["b." + f].cpu().numpy()
    for f, _dt, _ in ROW_COLUMNS:
        out.rows[f][:] = dev["r." + f].cpu().numpy()
    return out


def unchanged(a, b):
    """Every column of two stage copies byte for byte, inputs and outputs alike."""
    for f, _dt, _ in BODY_COLUMNS:
        if a.body[f].tobytes() != b.body[f].tobytes():
            return f"body {f}"
    for f, _dt, _ in ROW_COLUMNS:
        if a.rows[f].tobytes() != b.rows[f].tobytes():
            return f"row {f}"
    return None


def finish_with(world, copy):
    B, R, _ = world.views()
    for f, _dt, per in BODY_COLUMNS:
        n = per * copy.capacity
        if n:
            np.ctypeslib.as_array(getattr(B, f), shape=(n,))[:] = copy.body[f]
    for f, _dt, per in ROW_COLUMNS:
        n = per * copy.count
        if n:
            np.ctypeslib.as_array(getattr(R, f), shape=(n,))[:] = copy.rows[f]
    world.end_step()


def two_calls_against_the_oracle(w):
    for call in range(2):
        w.begin_step(DT)
        base = StageCopy(w)
        assert 0 < base.count <= _ffi.BG_STATIC_MAX_ROWS and base.capacity <= _ffi.BG_STATIC_MAX_BODIES
        want = oracle_io.solve(base.copy())
        got = solve_static(base.copy())
        assert first_difference(want, got) is None, f"call {call + 1}: {first_difference(want, got)}"
        finish_with(w, want)
    return base


def test_static_entry_point_matches_the_oracle_on_two_calls_in_a_row():
    w = World({}, solver=oracle_io.solver(0))
    scenes.pyramid(w, rows=8)
    w.addBody({"shape": "sphere", "radius": 0.4, "restitution": 0.5, "position": (6.0, 2.0, 0.0)})
    for _ in range(3):
        w.step(DT)
    two_calls_against_the_oracle(w)


def test_static_entry_point_at_its_limits():
    # 507 mixed bodies and five static walls (512 slots, the most it takes) heaped in a 6 m pen:
    # ~1,850 rows in 17 colours by step 240, against the 2,048 the fixed array holds.
    w = World({}, solver=oracle_io.solver(0))
    scenes.pile(w, count=507, seed=7, extent=6.0)
    for _ in range(240):
        w.step(DT)
    base = two_calls_against_the_oracle(w)
    assert base.capacity == _ffi.BG_STATIC_MAX_BODIES and base.count > 1800, (base.capacity, base.count)


def test_static_entry_point_refuses_bad_input_and_writes_nothing():
    w = World({}, solver=oracle_io.solver(0))
    scenes.pyramid(w, rows=8)
    for _ in range(3):
        w.step(DT)
    w.begin_step(DT)
    base = StageCopy(w)
    assert base.solved > 2
    for bad in ("starts", "a", "points", "row", "row twice", "awake"):
        work = base.copy()
        if bad == "starts":
            work.starts[1] = work.starts[2] + 1                    # colour starts must not decrease
        elif bad == "a":
            work.rows["a"][1] = work.capacity                      # not a slot
        elif bad == "points":
            work.rows["points"][0] = 5                             # 1..4
        elif bad == "row":
            work.rows["row"][0] = work.count                       # not a row
        elif bad == "row twice":
            work.rows["row"][1] = work.rows["row"][0]              # not a permutation
        else:
            work.awake_list[0] = -1                                # not a slot
        got = solve_static(work, expect=_ffi.BG_EINVAL)
        assert unchanged(work, got) is None, f"{bad}: {unchanged(work, got)}"
    # and the next good call is exact
    assert first_difference(oracle_io.solve(base.copy()), solve_static(base.copy())) is None


def test_static_entry_point_refuses_a_world_past_its_limit():
    w = World({}, solver=oracle_io.solver(0))
    scenes.pyramid(w, rows=8)
    w.begin_step(DT)
    base = StageCopy(w)
    B, R, S = base.views()
    B.capacity = _ffi.BG_STATIC_MAX_BODIES + 1
    assert _ffi.gpu().bg_solve_step_static(C.byref(B), C.byref(R), C.byref(S), None) == _ffi.BG_EINVAL
