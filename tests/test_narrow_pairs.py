"""The pair list a step's narrowphase worked on (bw_narrow_pairs) and the host's narrowphase over
such a list (bw_collide_pairs), on the CPU: run over the list the world recorded, the narrowphase
finds exactly the manifolds the world emitted as rows (their count, normal, points and
separations, in found order), so the list is the narrowphase's whole input and the device
narrowphase (bg_collide) can be checked against it pair by pair."""
import ctypes as C

import numpy as np
import pytest

import narrow_io
import oracle_io
from stage_io import StageCopy
from bearing_b200 import _ffi, scenes
from bearing_b200.world import World

DT = 1 / 60
P = _ffi.BG_POINTS


def boxes_and_balls(w):
    scenes.pile(w, count=600, seed=7, extent=10.0)


def raining(w):
    scenes.rain(w, count=150, seed=3)


@pytest.mark.parametrize("build,steps", [(scenes.pyramid, 10), (boxes_and_balls, 40), (raining, 90)],
                         ids=["pyramid", "pile600", "rain150"])
def test_the_recorded_pairs_give_the_worlds_rows(build, steps):
    w = World({}, solver=oracle_io.solver(0))
    build(w)
    for _ in range(steps):
        w.step(DT)
    w.begin_step(DT)
    pairs = narrow_io.world_pairs(w)
    assert pairs.count > 0
    B, R, S = w.views()
    got = narrow_io.host_collide(B, tuple(S.gravity), pairs)
    rows = StageCopy(w)
    met = np.flatnonzero(got.points[: pairs.count] > 0)
    assert met.size == rows.count   # every met pair is a row, in found order
    for f, i in enumerate(met):
        m = int(rows.rows["row"][f])
        n = int(got.points[i])
        assert rows.rows["points"][m] == n
        assert rows.rows["a"][m] == pairs.a[i] and rows.rows["b"][m] == pairs.b[i]
        assert got.normal[3 * i: 3 * i + 3].tobytes() == rows.rows["normal"][3 * m: 3 * m + 3].tobytes()
        assert got.separation[P * i: P * i + n].tobytes() == rows.rows["separation"][P * m: P * m + n].tobytes()
        assert got.point[3 * P * i: 3 * P * i + 3 * n].tobytes() == \
            rows.rows["point"][3 * P * m: 3 * P * m + 3 * n].tobytes()
    # a pair with no contact leaves zeros, as do the entries past a manifold's points
    empty = got.points[: pairs.count] == 0
    assert not got.normal[: 3 * pairs.count].reshape(-1, 3)[empty].any()
    counts = got.points[: pairs.count].astype(np.int64)
    unused = np.arange(P)[None, :] >= counts[:, None]
    assert not got.separation[: P * pairs.count].reshape(-1, P)[unused].any()
    assert not got.pid[: P * pairs.count].reshape(-1, P)[unused].any()
    w.destroy()


def test_bad_slots_are_refused():
    w = World({}, solver=oracle_io.solver(0))
    scenes.pyramid(w, rows=3)
    w.begin_step(DT)
    pairs = narrow_io.world_pairs(w)
    B, _, S = w.views()
    pairs.b[0] = B.capacity
    out = narrow_io.ManifoldSet(pairs.count)
    g = np.zeros(3)
    rc = _ffi.host().bw_collide_pairs(C.byref(B), g.ctypes.data_as(C.POINTER(C.c_double)), C.byref(pairs.view()),
                                      C.byref(out.s), 1)
    assert rc == _ffi.BG_EINVAL
    w.destroy()


NARROWPHASE = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.POINTER(_ffi.Bodies), C.POINTER(C.c_double),
                          C.POINTER(_ffi.Pairs), C.POINTER(_ffi.Manifolds))


@pytest.mark.parametrize("reuse", [False, True], ids=["fresh", "reuse"])
@pytest.mark.parametrize("build,steps", [(boxes_and_balls, 60), (raining, 100)], ids=["pile600", "rain150"])
def test_a_world_with_its_narrowphase_handed_out_is_the_same_world(build, steps, reuse):
    # bw_set_narrowphase with the host's own narrowphase behind it (what bg_collide computes on
    # the device, bit for bit): the two-pass walk over the pairs gives the same world, step by step,
    # with the kept-manifold cache on as well (the pairs that keep theirs are not handed out).
    host = _ffi.host()
    calls = []

    def collide(user, bodies, gravity, pairs, out):
        calls.append(pairs.contents.count)
        return host.bw_collide_pairs(bodies, gravity, pairs, out, 2)

    hook = NARROWPHASE(collide)
    a = World({"reuse": reuse}, solver=oracle_io.solver(0))
    b = World({"reuse": reuse}, solver=oracle_io.solver(0))
    build(a)
    build(b)
    assert host.bw_set_narrowphase(b._w, C.cast(hook, C.c_void_p), None) == 0
    for i in range(steps):
        a.step(DT)
        b.step(DT)
        sa, sb = a.state(), b.state()
        for k in ("position", "rotation", "velocity", "angular"):
            assert sa[k].tobytes() == sb[k].tobytes(), f"step {i + 1}: {k}"
    assert len(calls) > 0 and max(calls) > 0
    assert a.stats()["rows"] == b.stats()["rows"]
    assert host.bw_set_narrowphase(b._w, None, None) == 0
    a.destroy()
    b.destroy()


def test_a_long_pair_list_is_marked_on_several_threads_with_the_same_result():
    # Past 131,072 pairs the walk's box comparisons run on several threads before the walk takes
    # the pairs in order: a 20,000-body pile falling reaches 200,000 pairs by step 50.
    host = _ffi.host()

    def collide(user, bodies, gravity, pairs, out):
        return host.bw_collide_pairs(bodies, gravity, pairs, out, 4)

    hook = NARROWPHASE(collide)
    a = World({}, solver=oracle_io.solver(0))
    b = World({}, solver=oracle_io.solver(0))
    for w in (a, b):
        scenes.pile(w, count=20_000, extent=60.0)
    assert host.bw_set_narrowphase(b._w, C.cast(hook, C.c_void_p), None) == 0
    most = 0
    for i in range(55):
        a.step(DT)
        b.step(DT)
        sa, sb = a.state(), b.state()
        for k in ("position", "rotation", "velocity", "angular"):
            assert sa[k].tobytes() == sb[k].tobytes(), f"step {i + 1}: {k}"
        assert a.stats()["pairs"] == b.stats()["pairs"]
        most = max(most, b.stats()["pairs"])
    assert most >= 2 * 65536
    assert host.bw_set_narrowphase(b._w, None, None) == 0
    a.destroy()
    b.destroy()


def test_the_pair_upkeep_is_the_same_on_one_thread_and_on_many():
    # World.workers sets the threads of the walk over the pairs (past 131,072 pairs); with none it
    # runs on the caller's thread alone, as the reference's World does with workers 0.  The
    # 20,000-body pile passes 200,000 pairs by step 50, with pairs dropped as it falls.
    host = _ffi.host()

    def collide(user, bodies, gravity, pairs, out):
        return host.bw_collide_pairs(bodies, gravity, pairs, out, 4)

    hook = NARROWPHASE(collide)
    one = World({"workers": 0}, solver=oracle_io.solver(0))
    many = World({"workers": 7}, solver=oracle_io.solver(0))
    for w in (one, many):
        scenes.pile(w, count=20_000, extent=60.0)
        assert host.bw_set_narrowphase(w._w, C.cast(hook, C.c_void_p), None) == 0
    for i in range(55):
        one.step(DT)
        many.step(DT)
        sa, sb = one.state(), many.state()
        for k in ("position", "rotation", "velocity", "angular"):
            assert sa[k].tobytes() == sb[k].tobytes(), f"step {i + 1}: {k}"
        assert one.stats() == many.stats()
        ca, cb = one.contacts(), many.contacts()
        assert all(ca[k].tobytes() == cb[k].tobytes() for k in ca), f"step {i + 1}: contacts"
    assert many.stats()["pairs"] >= 2 * 65536
    for w in (one, many):
        assert host.bw_set_narrowphase(w._w, None, None) == 0
        w.destroy()
    assert host.bw_set_workers(None, 0) == _ffi.BG_EINVAL


def test_a_failing_narrowphase_fails_the_step():
    host = _ffi.host()
    hook = NARROWPHASE(lambda *args: _ffi.BG_ECUDA)
    w = World({}, solver=oracle_io.solver(0))
    scenes.pyramid(w, rows=3)
    assert host.bw_set_narrowphase(w._w, C.cast(hook, C.c_void_p), None) == 0
    assert host.bw_begin_step(w._w, DT) == _ffi.BG_ECUDA
    assert host.bw_set_narrowphase(w._w, None, None) == 0
    w.destroy()
