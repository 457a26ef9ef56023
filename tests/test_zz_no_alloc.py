"""bg_solve_step_static, the entry point that allocates nothing, against bg_solve_step.

It is for callers that cannot allocate device memory themselves: a host runtime that owns every
device buffer in a pool of its own and passes this library only pointers into it, or a per-frame
loop that must not take a cudaMalloc's synchronisation.  Such a caller passes device arrays;
here torch stands in for the caller's pool.  The result must be bit-identical to bg_solve_step's
on the same input, on two calls in a row (the second sees the first's leftovers in the library's
fixed working array, which it must not depend on).  Named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import gpu_io
import oracle_io
from stage_io import BODY_COLUMNS, ROW_COLUMNS, StageCopy, first_difference
from bearing_b200 import _ffi, scenes
from bearing_b200.world import World

pytestmark = pytest.mark.gpu

DT = 1 / 60
_CT = {np.float64: C.c_double, np.uint8: C.c_uint8, np.int32: C.c_int32}


def solve_static(copy):
    """Runs `copy` through bg_solve_step_static with every array in device memory."""
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
    assert rc == _ffi.BG_OK, f"bg_solve_step_static returned {rc}"
    torch.cuda.synchronize()
    out = copy.copy()
    for f, _dt, _ in BODY_COLUMNS:
        out.body[f][:] = dev["b." + f].cpu().numpy()
    for f, _dt, _ in ROW_COLUMNS:
        out.rows[f][:] = dev["r." + f].cpu().numpy()
    return out


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


def test_static_entry_point_matches_bg_solve_step_on_two_calls_in_a_row():
    w = World({}, solver=oracle_io.solver(0))
    scenes.pyramid(w, rows=8)
    w.addBody({"shape": "sphere", "radius": 0.4, "restitution": 0.5, "position": (6.0, 2.0, 0.0)})
    for _ in range(3):
        w.step(DT)
    for call in range(2):
        w.begin_step(DT)
        base = StageCopy(w)
        assert 0 < base.count <= _ffi.BG_STATIC_MAX_ROWS and base.capacity <= _ffi.BG_STATIC_MAX_BODIES
        want = gpu_io.solve(base.copy())
        got = solve_static(base.copy())
        assert first_difference(want, got) is None, f"call {call + 1}: {first_difference(want, got)}"
        finish_with(w, want)


def test_static_entry_point_refuses_a_world_past_its_limit():
    w = World({}, solver=oracle_io.solver(0))
    scenes.pyramid(w, rows=8)
    w.begin_step(DT)
    base = StageCopy(w)
    B, R, S = base.views()
    B.capacity = _ffi.BG_STATIC_MAX_BODIES + 1
    assert _ffi.gpu().bg_solve_step_static(C.byref(B), C.byref(R), C.byref(S), None) == _ffi.BG_EINVAL
