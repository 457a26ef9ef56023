"""Edge cases of the C ABI on the GPU: an empty world, a refused input that must write nothing,
and a ragged batch (worlds with no rows, no awake bodies, or a lone body) on every path."""
import ctypes as C

import numpy as np
import pytest

import gpu_io
import oracle_io
from stage_io import BatchCopy, StageCopy, first_difference
from bearing_b200 import _ffi, scenes
from bearing_b200.world import World

pytestmark = pytest.mark.gpu

DT = 1 / 60


def test_an_empty_world():
    w = World({}, solver=oracle_io.solver(0))
    w.begin_step(DT)
    base = StageCopy(w)
    assert base.capacity == 0 and base.count == 0
    a = oracle_io.solve(base.copy())
    b = gpu_io.solve(base.copy())
    assert first_difference(a, b) is None


# Inputs bg_solve_step must refuse before any kernel reads them: counts and colour starts, and
# every index the caller hands over (a row's bodies, its point count, the found order, the awake
# list), each of which would otherwise address memory outside the world.
BAD_INPUTS = ("starts", "solved", "awake count", "a", "b", "points", "row", "row twice", "awake list")


def spoil(work, bad, row0=0, body_count=None):
    n = work.capacity if body_count is None else body_count
    if bad == "starts":
        work.starts[1] = work.starts[2] + 1                 # colour starts must not decrease
    elif bad == "solved":
        work.solved = work.count + 1
    elif bad == "awake count":
        work.awake_count = work.capacity + 1
    elif bad == "a":
        work.rows["a"][row0 + 1] = n                        # one past the world's slots
    elif bad == "b":
        work.rows["b"][row0 + 2] = -1
    elif bad == "points":
        work.rows["points"][row0] = 0                       # 1..4
    elif bad == "row":
        work.rows["row"][row0 + 3] = 1 << 20                # not a row of the world
    elif bad == "row twice":
        work.rows["row"][row0 + 1] = work.rows["row"][row0]  # not a permutation
    else:
        work.awake_list[-1] = n


def unchanged(a, b):
    """Every column of two stage copies byte for byte, inputs and outputs alike."""
    for f, v in a.body.items():
        if v.tobytes() != b.body[f].tobytes():
            return f"body {f}"
    for f, v in a.rows.items():
        if v.tobytes() != b.rows[f].tobytes():
            return f"row {f}"
    return None if a.awake_list.tobytes() == b.awake_list.tobytes() else "awake_list"


def test_a_refused_world_writes_nothing():
    w = World({}, solver=oracle_io.solver(0))
    scenes.pyramid(w, rows=6)
    for _ in range(5):
        w.step(DT)
    w.begin_step(DT)
    base = StageCopy(w)
    assert base.solved > 0
    g = _ffi.gpu()
    ctx = g.bg_create(0, 0)
    try:
        for bad in BAD_INPUTS:
            work = base.copy()
            spoil(work, bad)
            before = work.copy()
            B, R, S = work.views()
            assert g.bg_solve_step(ctx, C.byref(B), C.byref(R), C.byref(S)) == _ffi.BG_EINVAL, bad
            assert g.bg_last_error(ctx).decode() != ""
            assert unchanged(before, work) is None, f"{bad}: {unchanged(before, work)}"
            # nothing stays uploaded from a refused call
            assert g.bg_restore(ctx) == _ffi.BG_EINVAL, bad
        # the context goes on
        work = base.copy()
        B, R, S = work.views()
        assert g.bg_solve_step(ctx, C.byref(B), C.byref(R), C.byref(S)) == 0, g.bg_last_error(ctx).decode()
        assert first_difference(oracle_io.solve(base.copy()), work) is None
    finally:
        g.bg_destroy(ctx)


def ragged_worlds():
    worlds = []
    for kind in range(6):
        w = World({}, solver=oracle_io.solver(0))
        if kind == 0:      # only a static ground: no awake body, no row
            w.addBody({"type": "static", "size": (10.0, 1.0, 10.0), "position": (0.0, -0.5, 0.0)})
        elif kind == 1:    # a lone falling body: awake, no row
            w.addBody({"position": (0.0, 20.0, 0.0), "angularVelocity": (0.5, 1.0, 0.0)})
        elif kind == 2:    # nothing at all
            pass
        else:              # the batch's own scenes
            scenes.batch_world(w, np.random.default_rng(100 + kind))
        worlds.append(w)
    for w in worlds:
        for _ in range(12):
            w.step(DT)
    return worlds


def test_a_ragged_batch_on_every_path():
    worlds = ragged_worlds()
    host = _ffi.host()
    handles = (C.c_void_p * len(worlds))(*[w._w for w in worlds])
    b = host.bw_batch_create(handles, len(worlds))
    try:
        assert host.bw_batch_begin_step(b, DT, 2) == 0
        B, R, W, S = _ffi.Bodies(), _ffi.Rows(), _ffi.Worlds(), _ffi.Step()
        assert host.bw_batch_views(b, C.byref(B), C.byref(R), C.byref(W), C.byref(S)) == 0
        base = BatchCopy(B, R, W, S)
    finally:
        host.bw_batch_destroy(b)
    counts = [(int(base.body_offset[i + 1] - base.body_offset[i]), int(base.row_offset[i + 1] - base.row_offset[i]))
              for i in range(base.worlds)]
    assert counts[0][1] == 0 and counts[1][1] == 0 and counts[2] == (0, 0)
    assert sum(r for _, r in counts) > 0
    want = [oracle_io.solve(base.world(i).copy()) for i in range(base.worlds)]
    g = _ffi.gpu()
    for threads, groups in ((32, 1), (256, 1), (_ffi.BG_BATCH_ON_GRID, 1), (0, 1), (0, 3)):
        ctx = g.bg_create(0, 0)
        try:
            assert g.bg_set_block_threads(ctx, threads) == 0
            assert g.bg_set_batch_groups(ctx, groups) == 0
            work = base.copy()
            Bw, Rw, Ww, Sw = work.views()
            rc = g.bg_batch_solve_step(ctx, C.byref(Bw), C.byref(Rw), C.byref(Ww), C.byref(Sw))
            assert rc == 0, g.bg_last_error(ctx).decode()
            for i in range(base.worlds):
                d = first_difference(want[i], work.world(i))
                assert d is None, f"{threads} threads, {groups} groups, world {i}: {d}"
        finally:
            g.bg_destroy(ctx)


def test_a_refused_batch_writes_nothing_on_any_path():
    # A bad index in the batch's last world: refused before any group runs, whether the batch goes
    # in one piece or in groups of worlds (where the first groups would otherwise have been solved
    # and written back already).
    worlds = ragged_worlds()
    host = _ffi.host()
    handles = (C.c_void_p * len(worlds))(*[w._w for w in worlds])
    b = host.bw_batch_create(handles, len(worlds))
    try:
        assert host.bw_batch_begin_step(b, DT, 2) == 0
        B, R, W, S = _ffi.Bodies(), _ffi.Rows(), _ffi.Worlds(), _ffi.Step()
        assert host.bw_batch_views(b, C.byref(B), C.byref(R), C.byref(W), C.byref(S)) == 0
        base = BatchCopy(B, R, W, S)
    finally:
        host.bw_batch_destroy(b)
    last = base.worlds - 1
    row0 = int(base.row_offset[last])
    nb = int(base.body_offset[last + 1] - base.body_offset[last])
    assert int(base.row_offset[last + 1]) - row0 > 4
    g = _ffi.gpu()
    for groups in (1, 3):
        for bad in ("a", "b", "points", "row", "row twice", "awake list"):
            ctx = g.bg_create(0, 0)
            try:
                assert g.bg_set_batch_groups(ctx, groups) == 0
                work = base.copy()
                spoil(work.stage, bad, row0=row0, body_count=nb)
                before = work.copy()
                Bw, Rw, Ww, Sw = work.views()
                rc = g.bg_batch_solve_step(ctx, C.byref(Bw), C.byref(Rw), C.byref(Ww), C.byref(Sw))
                assert rc == _ffi.BG_EINVAL, f"{groups} groups, {bad}: {rc}"
                assert unchanged(before.stage, work.stage) is None, f"{groups} groups, {bad}"
            finally:
                g.bg_destroy(ctx)
