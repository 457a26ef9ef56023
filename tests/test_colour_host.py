"""The colouring's checkers on the CPU: the plain restatement of src/graph.js:105-166
(colour_io.reference_colour) against the World's own colouring of its manifolds, and the host's
colouring over any manifold list (bw_colour_rows, what bg_colour computes on the device) against
both."""
import ctypes as C

import numpy as np
import pytest

import oracle_io
from colour_io import made_up_manifolds, reference_colour
from stage_io import StageCopy
from bearing_b200 import _ffi, scenes
from bearing_b200.world import World

DT = 1 / 60
_PI = C.POINTER(C.c_int32)


def host_colour(type_, frozen, a, b):
    n, nb = len(a), len(type_)
    B = _ffi.Bodies()
    B.capacity = nb
    t = np.ascontiguousarray(type_, np.uint8)
    fz = np.ascontiguousarray(frozen, np.uint8)
    B.type = t.ctypes.data_as(C.POINTER(C.c_uint8))
    B.frozen = fz.ctypes.data_as(C.POINTER(C.c_uint8))
    a = np.ascontiguousarray(a, np.int32)
    b = np.ascontiguousarray(b, np.int32)
    colour = np.zeros(max(n, 1), np.int32)
    order = np.zeros(max(n, 1), np.int32)
    starts = np.zeros(_ffi.BG_STARTS, np.int32)
    solved = C.c_int32(-1)
    rc = _ffi.host().bw_colour_rows(C.byref(B), n, a.ctypes.data_as(_PI), b.ctypes.data_as(_PI),
                                    colour.ctypes.data_as(_PI), order.ctypes.data_as(_PI),
                                    starts.ctypes.data_as(_PI), C.byref(solved))
    return rc, colour[:n], order[:n], starts, solved.value


def slab(w):
    # a dynamic slab carrying 49 boxes: more manifolds on one body than there are colours
    w.addBody({"type": "static", "size": (40.0, 1.0, 40.0), "position": (0.0, -0.5, 0.0)})
    w.addBody({"size": (8.0, 0.5, 8.0), "position": (0.0, 0.25, 0.0)})
    for i in range(7):
        for j in range(7):
            w.addBody({"size": (0.8, 0.8, 0.8), "position": (-3.0 + i, 0.9, -3.0 + j)})


def pile600(w):
    scenes.pile(w, count=600, seed=7, extent=10.0)


@pytest.mark.parametrize("build,steps", [(scenes.pyramid, 10), (slab, 5), (pile600, 40)],
                         ids=["pyramid", "slab49", "pile600"])
def test_the_restatement_and_the_host_colour_a_world_as_it_did(build, steps):
    w = World({}, solver=oracle_io.solver(0))
    build(w)
    for _ in range(steps):
        w.step(DT)
    w.begin_step(DT)
    copy = StageCopy(w)
    w.destroy()
    n = copy.count
    row = copy.rows["row"][:n]
    a, b = copy.rows["a"][row], copy.rows["b"][row]
    found = np.empty(n, np.int32)
    found[row] = np.arange(n, dtype=np.int32)   # row o holds the manifold found found[o]-th
    colour, order, starts, solved = reference_colour(copy.body["type"], copy.body["frozen"], a, b)
    assert np.array_equal(order, found) and np.array_equal(starts, copy.starts) and solved == copy.solved
    rc, colour2, order2, starts2, solved2 = host_colour(copy.body["type"], copy.body["frozen"], a, b)
    assert rc == 0
    assert np.array_equal(colour2, colour) and np.array_equal(order2, order)
    assert np.array_equal(starts2, starts) and solved2 == solved
    if build is slab:
        assert starts[33] > starts[32]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_the_host_colours_made_up_manifolds_as_the_restatement(seed):
    type_, frozen, a, b = made_up_manifolds(seed)
    want = reference_colour(type_, frozen, a, b)
    rc, colour, order, starts, solved = host_colour(type_, frozen, a, b)
    assert rc == 0
    assert np.array_equal(colour, want[0]) and np.array_equal(order, want[1])
    assert np.array_equal(starts, want[2]) and solved == want[3]
    assert starts[33] > starts[32] and starts[34] > starts[33]


def test_bad_slots_are_refused():
    z = np.zeros(4, np.uint8)
    assert host_colour(z, z, [0, 1], [1, 4])[0] == _ffi.BG_EINVAL
    assert host_colour(z, z, [2], [2])[0] == _ffi.BG_EINVAL
