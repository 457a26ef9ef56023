"""A batch's input cut down to some of its worlds (stage_io.BatchCopy.subset, which the benchmark's
size-class split uses): each world of the subset is the batch's own, column for column, and all of
them in order give the batch back.  On the CPU, with the host library's batch views."""
import ctypes as C

import numpy as np

import oracle_io
from stage_io import BODY_COLUMNS, ROW_COLUMNS, BatchCopy
from bearing_b200 import _ffi, scenes
from bearing_b200.world import World

DT = 1 / 60


def a_batch(count=9, steps=20):
    worlds = []
    for i in range(count):
        w = World({}, solver=oracle_io.solver(0))
        scenes.batch_world(w, scenes.batch_rng(5, i))
        for _ in range(steps):
            w.step(DT)
        worlds.append(w)
    lib = _ffi.host()
    arr = (C.c_void_p * count)(*[w._w for w in worlds])
    b = lib.bw_batch_create(arr, count)
    assert b and lib.bw_batch_begin_step(b, DT, 2) == 0
    B, R, W, S = _ffi.Bodies(), _ffi.Rows(), _ffi.Worlds(), _ffi.Step()
    assert lib.bw_batch_views(b, C.byref(B), C.byref(R), C.byref(W), C.byref(S)) == 0
    copy = BatchCopy(B, R, W, S)
    lib.bw_batch_destroy(b)
    for w in worlds:
        w.destroy()
    return copy


def same_world(x, y):
    assert x.capacity == y.capacity and x.count == y.count and x.solved == y.solved
    assert np.array_equal(x.starts, y.starts) and np.array_equal(x.awake_list, y.awake_list)
    for f, _, _ in BODY_COLUMNS:
        assert x.body[f].tobytes() == y.body[f].tobytes(), f
    for f, _, _ in ROW_COLUMNS:
        assert x.rows[f].tobytes() == y.rows[f].tobytes(), f


def test_a_subset_holds_the_batchs_own_worlds():
    base = a_batch()
    pick = [7, 2, 4]
    sub = base.subset(pick)
    assert sub.worlds == 3
    for j, i in enumerate(pick):
        same_world(sub.world(j), base.world(i))


def test_every_world_in_order_gives_the_batch_back():
    base = a_batch()
    whole = base.subset(range(base.worlds))
    for k in ("body_offset", "awake_offset", "row_offset", "starts"):
        assert np.array_equal(getattr(whole, k), getattr(base, k)), k
    for f, _, _ in BODY_COLUMNS:
        assert whole.stage.body[f].tobytes() == base.stage.body[f].tobytes(), f
    for f, _, _ in ROW_COLUMNS:
        assert whole.stage.rows[f].tobytes() == base.stage.rows[f].tobytes(), f
    assert np.array_equal(whole.stage.awake_list, base.stage.awake_list)


def test_save_and_load_give_the_batch_back(tmp_path):
    base = a_batch(count=4)
    base.save(tmp_path / "b")
    back = BatchCopy.load(tmp_path / "b")
    assert back.worlds == base.worlds
    for k in ("body_offset", "awake_offset", "row_offset", "starts"):
        assert np.array_equal(getattr(back, k), getattr(base, k)), k
    for i in range(base.worlds):
        same_world(back.world(i), base.world(i))
