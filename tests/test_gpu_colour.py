"""The colouring on the device (bg_colour) against the host's (the World's own colour() and
arrange(), src/graph.js:105-214) and against a plain restatement of graph.js over made-up
manifold lists with static, kinematic and frozen bodies, the overflow colour and the resting run:
every colour, the row order and the colour starts, exactly."""
import ctypes as C

import numpy as np
import pytest

import oracle_io
from colour_io import made_up_manifolds, reference_colour
from stage_io import StageCopy
from bearing_b200 import _ffi, scenes
from bearing_b200.world import GpuSolver, World

pytestmark = pytest.mark.gpu

DT = 1 / 60
_PI = C.POINTER(C.c_int32)
_ctx = {}


def ctx():
    if "c" not in _ctx:
        _ctx["c"] = _ffi.gpu().bg_create(0, 0)
        assert _ctx["c"]
    return _ctx["c"]


def device_colour(type_, frozen, a, b):
    n, nb = len(a), len(type_)
    B = _ffi.Bodies()
    B.capacity = nb
    t = np.ascontiguousarray(type_, np.uint8)
    fz = np.ascontiguousarray(frozen, np.uint8)
    B.type = t.ctypes.data_as(C.POINTER(C.c_uint8))
    B.frozen = fz.ctypes.data_as(C.POINTER(C.c_uint8))
    a = np.ascontiguousarray(a, np.int32)
    b = np.ascontiguousarray(b, np.int32)
    colour = np.full(max(n, 1), -7, np.int32)
    order = np.full(max(n, 1), -7, np.int32)
    starts = np.zeros(_ffi.BG_STARTS, np.int32)
    solved = C.c_int32(-1)
    lib = _ffi.gpu()
    rc = lib.bg_colour(ctx(), C.byref(B), n, a.ctypes.data_as(_PI), b.ctypes.data_as(_PI), colour.ctypes.data_as(_PI),
                       order.ctypes.data_as(_PI), starts.ctypes.data_as(_PI), C.byref(solved))
    return rc, colour[:n], order[:n], starts, solved.value


def world_input(build, steps):
    w = World({}, solver=oracle_io.solver(0))
    build(w)
    for _ in range(steps):
        w.step(DT)
    w.begin_step(DT)
    copy = StageCopy(w)
    w.destroy()
    return copy


def slab(w):
    # a dynamic slab carrying 49 boxes: more manifolds on one body than there are colours
    w.addBody({"type": "static", "size": (40.0, 1.0, 40.0), "position": (0.0, -0.5, 0.0)})
    w.addBody({"size": (8.0, 0.5, 8.0), "position": (0.0, 0.25, 0.0)})
    for i in range(7):
        for j in range(7):
            w.addBody({"size": (0.8, 0.8, 0.8), "position": (-3.0 + i, 0.9, -3.0 + j)})


def pile2000(w):
    scenes.pile(w, count=2000, seed=9, extent=14.0)


def check_against_the_world(copy):
    n = copy.count
    row = copy.rows["row"][:n]
    a, b = copy.rows["a"][row], copy.rows["b"][row]   # the manifolds in found order
    rc, colour, order, starts, solved = device_colour(copy.body["type"], copy.body["frozen"], a, b)
    assert rc == 0, _ffi.gpu().bg_last_error(ctx())
    found = np.empty(n, np.int32)
    found[row] = np.arange(n, dtype=np.int32)   # the host's c.order: row o holds found[o]
    assert np.array_equal(order, found)
    assert np.array_equal(starts, copy.starts)
    assert solved == copy.solved
    run = np.searchsorted(copy.starts[:34], row, side="right") - 1   # each found manifold's run
    assert np.array_equal(colour, run)
    return starts


@pytest.mark.parametrize("build,steps", [(scenes.pyramid, 20), (slab, 5), (pile2000, 80)],
                         ids=["pyramid", "slab49", "pile2000"])
def test_the_device_colours_a_worlds_manifolds_as_the_host_does(build, steps):
    starts = check_against_the_world(world_input(build, steps))
    if build is slab:
        assert starts[33] > starts[32]   # the overflow holds manifolds


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_the_device_colours_made_up_manifolds_as_graph_js_does(seed):
    # static (1), kinematic (2) and frozen bodies, a hub body with 40 manifolds (overflow), and
    # pairs between frozen and static bodies (the resting run)
    type_, frozen, a, b = made_up_manifolds(seed)
    want = reference_colour(type_, frozen, a, b)
    rc, colour, order, starts, solved = device_colour(type_, frozen, a, b)
    assert rc == 0
    assert np.array_equal(colour, want[0])
    assert np.array_equal(order, want[1])
    assert np.array_equal(starts, want[2])
    assert solved == want[3]
    assert starts[33] > starts[32] and starts[34] > starts[33]   # overflow and resting rows present


def test_bad_slots_and_no_manifolds():
    type_ = np.zeros(4, np.uint8)
    frozen = np.zeros(4, np.uint8)
    assert device_colour(type_, frozen, [0, 1], [1, 4])[0] == _ffi.BG_EINVAL
    assert device_colour(type_, frozen, [2], [2])[0] == _ffi.BG_EINVAL
    rc, _, _, starts, solved = device_colour(type_, frozen, [], [])
    assert rc == 0 and solved == 0 and not starts.any()


def test_the_50k_pile_colours_as_the_host_does():
    w = World({}, solver=GpuSolver())
    w.set_narrowphase(w._solver)
    scenes.pile(w, count=50_000, seed=50_000)
    for _ in range(100):
        w.step(DT)
    w.begin_step(DT)
    check_against_the_world(StageCopy(w))
    assert _ffi.gpu().bg_last_colour_ms(ctx()) > 0
    w.destroy()


def test_a_static_body_under_ten_thousand_manifolds_of_one_colour():
    # The ground added last, so it is b (the higher slot) of every pair it is in: 10,000 boxes
    # resting on it put 10,000 manifolds of one colour on one (colour, b) key.  The order keeps
    # found order within it, and the sort costs what any other does.
    def build(w):
        for i in range(100):
            for j in range(100):
                w.addBody({"size": (0.8, 0.8, 0.8), "position": (i - 49.5, 0.4, j - 49.5)})
        w.addBody({"type": "static", "size": (120.0, 1.0, 120.0), "position": (0.0, -0.5, 0.0)})
    copy = world_input(build, 3)
    assert copy.count >= 10_000
    check_against_the_world(copy)
    assert 0 < _ffi.gpu().bg_last_colour_ms(ctx()) < 5.0
