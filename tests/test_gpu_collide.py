"""The device narrowphase (bg_collide) against the host's (bw_collide_pairs, the narrowphase the
step itself runs), bit for bit, on the pairs a step's narrowphase worked on: every pair's point
count, normal, points, separations and feature ids, and the zeros past each manifold's points."""
import ctypes as C

import numpy as np
import pytest

import narrow_io
import oracle_io
from bearing_b200 import _ffi, scenes
from bearing_b200.world import GpuSolver, World

pytestmark = pytest.mark.gpu

DT = 1 / 60
_ctx = {}


def ctx():
    if "c" not in _ctx:
        _ctx["c"] = _ffi.gpu().bg_create(0, 0)
        assert _ctx["c"]
    return _ctx["c"]


def device_collide(bodies, gravity, pairs):
    out = narrow_io.ManifoldSet(pairs.count, fill=0xCD)
    g = np.asarray(gravity, np.float64)
    lib = _ffi.gpu()
    rc = lib.bg_collide(ctx(), C.byref(bodies), g.ctypes.data_as(C.POINTER(C.c_double)), C.byref(pairs.view()),
                        C.byref(out.s))
    assert rc == 0, f"bg_collide: {rc} {lib.bg_last_error(ctx()).decode()}"
    return out


def check(world):
    world.begin_step(DT)
    pairs = narrow_io.world_pairs(world)
    B, _, S = world.views()
    want = narrow_io.host_collide(B, tuple(S.gravity), pairs, threads=8)
    got = device_collide(B, tuple(S.gravity), pairs)
    assert narrow_io.first_unequal(want, got) is None, narrow_io.first_unequal(want, got)
    return pairs, want


def pile600(w):
    scenes.pile(w, count=600, seed=7, extent=10.0)


def pile3000(w):
    scenes.pile(w, count=3000, seed=3, extent=20.0)


def rain(w):
    scenes.rain(w, count=300, seed=5)


@pytest.mark.parametrize("build,steps", [(scenes.pyramid, 0), (scenes.pyramid, 30), (pile600, 0), (pile600, 45),
                                         (pile3000, 120), (rain, 100), (scenes.stack, 20)],
                         ids=["pyramid0", "pyramid30", "pile600_0", "pile600_45", "pile3000", "rain300", "stack"])
def test_device_narrowphase_matches_the_host(build, steps):
    w = World({}, solver=oracle_io.solver(0))
    build(w)
    for _ in range(steps):
        w.step(DT)
    pairs, want = check(w)
    assert pairs.count > 0 and (want.points[: pairs.count] > 0).any()
    w.destroy()


def test_the_50k_pile_pairs_match_the_host():
    # The headline pile, stepped on the GPU, at step 151: about 260,000 pairs whose boxes meet,
    # boxes, spheres and capsules in every combination.
    w = World({}, solver=GpuSolver())
    scenes.pile(w, count=50_000, seed=50_000)
    for _ in range(150):
        w.step(DT)
    pairs, want = check(w)
    counts = np.bincount(want.points[: pairs.count], minlength=5)
    assert pairs.count > 200_000 and counts[1:].sum() > 100_000, counts
    assert (counts[1:] > 0).all()   # manifolds of 1, 2, 3 and 4 points
    w.destroy()


def test_refusals_write_nothing():
    w = World({}, solver=oracle_io.solver(0))
    scenes.pyramid(w, rows=3)
    w.begin_step(DT)
    pairs = narrow_io.world_pairs(w)
    B, _, S = w.views()
    g = np.asarray(S.gravity, np.float64)
    lib = _ffi.gpu()
    pairs.a[1] = -1
    out = narrow_io.ManifoldSet(pairs.count, fill=0x5A)
    rc = lib.bg_collide(ctx(), C.byref(B), g.ctypes.data_as(C.POINTER(C.c_double)), C.byref(pairs.view()),
                        C.byref(out.s))
    assert rc == _ffi.BG_EINVAL
    assert (out.points == 0x5A).all() and (out.pid == 0x5A).all()
    # no pairs: nothing to do
    empty = narrow_io.PairList(_ffi.Pairs())
    rc = lib.bg_collide(ctx(), C.byref(B), g.ctypes.data_as(C.POINTER(C.c_double)), C.byref(empty.view()),
                        C.byref(out.s))
    assert rc == 0
    w.destroy()


@pytest.mark.parametrize("reuse", [False, True], ids=["fresh", "reuse"])
@pytest.mark.parametrize("build,steps", [(pile3000, 60), (rain, 80)], ids=["pile3000", "rain300"])
def test_a_world_stepping_with_the_device_narrowphase_is_the_same_world(build, steps, reuse):
    # bw_set_narrowphase: each step's pairs go to bg_collide, and the step emits and carries its
    # manifolds; the state after every step equals the host narrowphase's, bit for bit, with the
    # kept-manifold cache on as well (the pairs that keep theirs stay on the host).
    a = World({"reuse": reuse}, solver=oracle_io.solver(0))
    b = World({"reuse": reuse}, solver=oracle_io.solver(0))
    build(a)
    build(b)
    device = GpuSolver()
    b.set_narrowphase(device)
    for i in range(steps):
        a.step(DT)
        b.step(DT)
        sa, sb = a.state(), b.state()
        for k in ("position", "rotation", "velocity", "angular"):
            assert sa[k].tobytes() == sb[k].tobytes(), f"step {i + 1}: {k}"
    assert a.stats()["rows"] == b.stats()["rows"] > 0
    b.set_narrowphase(None)
    a.destroy()
    b.destroy()
    device.close()
