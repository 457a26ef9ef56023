"""Batched worlds on the GPU (one launch, one CTA a world) against the oracle, world by world."""
import numpy as np
import pytest

import oracle_io
from bearing_b200 import scenes
from bearing_b200.world import Batch, World

pytestmark = pytest.mark.gpu

DT = 1 / 60


def make(n, seed, solver):
    rng = np.random.default_rng(seed)
    worlds = []
    for _ in range(n):
        w = World({}, solver=solver)
        scenes.batch_world(w, rng)
        worlds.append(w)
    return worlds


def test_batched_worlds_match_the_oracle_world_by_world():
    gpu_worlds = make(48, 17, oracle_io.solver(0))
    ref_worlds = make(48, 17, oracle_io.solver(0))
    batch = Batch(gpu_worlds, threads=4)
    for step in range(40):
        batch.step(DT)
        for w in ref_worlds:
            w.step(DT)
    for i, (a, b) in enumerate(zip(gpu_worlds, ref_worlds)):
        sa, sb = a.state(), b.state()
        for k in sa:
            assert sa[k].tobytes() == sb[k].tobytes(), f"world {i}: {k}"
    assert sum(w.stats()["rows"] for w in gpu_worlds) > 1000
    batch.destroy()


def test_batched_results_do_not_depend_on_the_cta_size():
    # 32, 64 and 256 threads a world, every world on the grid as one flow, and the tuner's own
    # choice: the same bits, the oracle's.
    import ctypes as C
    from stage_io import BatchCopy, first_difference
    from bearing_b200 import _ffi
    worlds = make(40, 23, oracle_io.solver(0))
    for w in worlds:
        for _ in range(25):
            w.step(DT)
    host = _ffi.host()
    handles = (C.c_void_p * len(worlds))(*[w._w for w in worlds])
    b = host.bw_batch_create(handles, len(worlds))
    try:
        assert host.bw_batch_begin_step(b, DT, 4) == 0
        B, R, W, S = _ffi.Bodies(), _ffi.Rows(), _ffi.Worlds(), _ffi.Step()
        assert host.bw_batch_views(b, C.byref(B), C.byref(R), C.byref(W), C.byref(S)) == 0
        base = BatchCopy(B, R, W, S)
    finally:
        host.bw_batch_destroy(b)
    g = _ffi.gpu()
    want = [oracle_io.solve(base.world(i).copy()) for i in range(base.worlds)]
    for threads in (32, 64, 256, _ffi.BG_BATCH_ON_GRID, 0):
        ctx = g.bg_create(0, 0)
        try:
            assert g.bg_set_block_threads(ctx, threads) == 0
            work = base.copy()
            Bw, Rw, Ww, Sw = work.views()
            rc = g.bg_batch_solve_step(ctx, C.byref(Bw), C.byref(Rw), C.byref(Ww), C.byref(Sw))
            assert rc == 0, g.bg_last_error(ctx).decode()
            used = g.bg_block_threads(ctx)
            assert used == threads if threads else used in (32, 64, 128, 256, _ffi.BG_BATCH_ON_GRID)
            for i in range(base.worlds):
                d = first_difference(want[i], work.world(i))
                assert d is None, f"{threads} threads, world {i}: {d}"
        finally:
            g.bg_destroy(ctx)
    assert g.bg_set_block_threads(None, 32) == _ffi.BG_EINVAL


def test_batch_in_groups_gives_the_same_bits():
    # bg_batch_solve_step split into groups of whole worlds, each copied in while the one before it
    # solves: every world's results are the oracle's whatever the split.
    import ctypes as C
    from stage_io import BatchCopy, first_difference
    from bearing_b200 import _ffi
    worlds = make(37, 29, oracle_io.solver(0))
    for w in worlds:
        for _ in range(20):
            w.step(DT)
    host = _ffi.host()
    handles = (C.c_void_p * len(worlds))(*[w._w for w in worlds])
    b = host.bw_batch_create(handles, len(worlds))
    try:
        assert host.bw_batch_begin_step(b, DT, 4) == 0
        B, R, W, S = _ffi.Bodies(), _ffi.Rows(), _ffi.Worlds(), _ffi.Step()
        assert host.bw_batch_views(b, C.byref(B), C.byref(R), C.byref(W), C.byref(S)) == 0
        base = BatchCopy(B, R, W, S)
    finally:
        host.bw_batch_destroy(b)
    g = _ffi.gpu()
    want = [oracle_io.solve(base.world(i).copy()) for i in range(base.worlds)]
    ctx = g.bg_create(0, 0)
    try:
        assert g.bg_set_batch_groups(ctx, _ffi.BG_MAX_BATCH_GROUPS + 1) == _ffi.BG_EINVAL
        assert g.bg_set_batch_groups(ctx, -1) == _ffi.BG_EINVAL
        for groups in (3, 1, 2, _ffi.BG_MAX_BATCH_GROUPS, 0, 5):
            assert g.bg_set_batch_groups(ctx, groups) == 0
            for rep in range(2):   # the second time through, each group's context is reused
                work = base.copy()
                Bw, Rw, Ww, Sw = work.views()
                rc = g.bg_batch_solve_step(ctx, C.byref(Bw), C.byref(Rw), C.byref(Ww), C.byref(Sw))
                assert rc == 0, g.bg_last_error(ctx).decode()
                for i in range(base.worlds):
                    d = first_difference(want[i], work.world(i))
                    assert d is None, f"{groups} groups, world {i}: {d}"
            if groups > 1:
                assert g.bg_restore(ctx) == _ffi.BG_EINVAL   # a split batch stays in its groups
        # A refused batch writes nothing, even when split: the last world's starts decrease.
        assert g.bg_set_batch_groups(ctx, 4) == 0
        work = base.copy()
        work.starts[_ffi.BG_STARTS * (base.worlds - 1) + 1] = -1
        before = work.copy()
        Bw, Rw, Ww, Sw = work.views()
        assert g.bg_batch_solve_step(ctx, C.byref(Bw), C.byref(Rw), C.byref(Ww), C.byref(Sw)) == _ffi.BG_EINVAL
        for i in range(base.worlds):
            assert first_difference(before.world(i), work.world(i)) is None
    finally:
        g.bg_destroy(ctx)
    assert g.bg_set_batch_groups(None, 2) == _ffi.BG_EINVAL


def test_a_batch_of_one_world_on_every_path():
    # One world given as a batch: each CTA size and the grid's batch flow solve it as the oracle does.
    import ctypes as C
    from stage_io import BatchCopy, first_difference
    from bearing_b200 import _ffi
    worlds = make(1, 31, oracle_io.solver(0))
    for _ in range(25):
        worlds[0].step(DT)
    host = _ffi.host()
    handles = (C.c_void_p * 1)(worlds[0]._w)
    b = host.bw_batch_create(handles, 1)
    try:
        assert host.bw_batch_begin_step(b, DT, 4) == 0
        B, R, W, S = _ffi.Bodies(), _ffi.Rows(), _ffi.Worlds(), _ffi.Step()
        assert host.bw_batch_views(b, C.byref(B), C.byref(R), C.byref(W), C.byref(S)) == 0
        base = BatchCopy(B, R, W, S)
    finally:
        host.bw_batch_destroy(b)
    assert int(base.starts[33]) > 0   # rows the solve moves
    want = oracle_io.solve(base.world(0).copy())
    g = _ffi.gpu()
    for threads in (32, 256, _ffi.BG_BATCH_ON_GRID, 0):
        ctx = g.bg_create(0, 0)
        try:
            assert g.bg_set_block_threads(ctx, threads) == 0
            work = base.copy()
            Bw, Rw, Ww, Sw = work.views()
            rc = g.bg_batch_solve_step(ctx, C.byref(Bw), C.byref(Rw), C.byref(Ww), C.byref(Sw))
            assert rc == 0, g.bg_last_error(ctx).decode()
            d = first_difference(want, work.world(0))
            assert d is None, f"{threads} threads: {d}"
        finally:
            g.bg_destroy(ctx)
