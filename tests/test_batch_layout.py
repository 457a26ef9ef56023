"""The batch's host side (bw_batch, include/bearing_world.h) lays every world's solve-stage input
end to end: world i's part of the batch views must be exactly what world i would pass alone.  Runs on
the CPU; the batched GPU solve itself is checked against the oracle in test_gpu_batch.py."""
import ctypes as C

import numpy as np

import oracle_io
from stage_io import BODY_COLUMNS, ROW_COLUMNS, BatchCopy, StageCopy
from bearing_b200 import _ffi, scenes
from bearing_b200.world import World

DT = 1 / 60


def test_each_worlds_part_of_the_batch_is_its_own_input():
    rng = np.random.default_rng(11)
    worlds = []
    for _ in range(10):
        w = World({}, solver=oracle_io.solver(0))
        scenes.batch_world(w, rng)
        for _ in range(15):
            w.step(DT)
        worlds.append(w)
    lib = _ffi.host()
    handles = (C.c_void_p * len(worlds))(*[w._w for w in worlds])
    b = lib.bw_batch_create(handles, len(worlds))
    assert b
    try:
        assert lib.bw_batch_begin_step(b, DT, 3) == 0
        B, R, W, S = _ffi.Bodies(), _ffi.Rows(), _ffi.Worlds(), _ffi.Step()
        assert lib.bw_batch_views(b, C.byref(B), C.byref(R), C.byref(W), C.byref(S)) == 0
        batch = BatchCopy(B, R, W, S)
        assert batch.worlds == len(worlds)
        rows = 0
        for i, w in enumerate(worlds):
            own, part = StageCopy(w), batch.world(i)
            assert (own.capacity, own.awake_count, own.count, own.solved) == \
                (part.capacity, part.awake_count, part.count, part.solved), f"world {i}"
            assert own.starts.tobytes() == part.starts.tobytes()
            assert own.awake_list.tobytes() == part.awake_list.tobytes()
            for f, _, _ in BODY_COLUMNS:
                assert own.body[f].tobytes() == part.body[f].tobytes(), f"world {i} body {f}"
            for f, _, _ in ROW_COLUMNS:
                assert own.rows[f].tobytes() == part.rows[f].tobytes(), f"world {i} rows {f}"
            rows += own.count
        assert rows > 100
    finally:
        lib.bw_batch_destroy(b)
