"""The kept-manifold cache (src/contact.js:388-595: reused, keeps, remember; src/pairs.js:55-80) in
the host's narrowphase, on the CPU, with World({"reuse": True}) as the reference always runs.

A settled stack and pyramid keep every manifold (no pair goes to the narrowphase) and stand and
sink as the reference's tests publish; a kept manifold's deepest point stays within the tolerance
of the one a fresh collide() finds, the bound REUSE's rules are built to hold; a pair moving fast
is found afresh; and a cloned world carries its cache with it."""
import ctypes as C
import math

import numpy as np
import pytest

import narrow_io
import oracle_io
from stage_io import StageCopy
from bearing_b200 import _ffi, scenes
from bearing_b200.world import World

DT = 1 / 60
P = _ffi.BG_POINTS


def world(reuse=True, workers=0):
    return World({"reuse": reuse}, solver=oracle_io.solver(workers))


def handed_to_collide(w):
    """Pairs the last begun step handed to collide() (the rest kept their manifolds)."""
    return narrow_io.world_pairs(w).count


def test_a_settled_stack_keeps_every_manifold_and_sinks_as_published():
    w = world()
    slots = scenes.stack(w, friction=0.5)[1:]
    for _ in range(600):
        w.step(DT)
    st = w.state()
    sank = 9.5 - st["position"][3 * slots[-1] + 1]
    assert abs(sank * 1000 - 6.9) < 0.1
    w.begin_step(DT)
    assert w.stats()["rows"] == 10 and handed_to_collide(w) == 0
    w.destroy()


def test_a_settled_pyramid_keeps_every_manifold_and_stands():
    # test/contact.test.js:45-64 with the reference's cache on, as it always runs.
    w = world()
    slots = scenes.pyramid(w, friction=0.5, ground_friction=0.5)[1:]
    start = w.state()["position"].copy()
    for _ in range(600):
        w.step(DT)
    st = w.state()
    stray = max(math.hypot(st["position"][3 * s] - start[3 * s], st["position"][3 * s + 2] - start[3 * s + 2])
                for s in slots)
    sank = start[3 * slots[-1] + 1] - st["position"][3 * slots[-1] + 1]
    assert stray * 1000 < 0.25 and abs(sank * 1000 - 7.4) < 0.1
    w.begin_step(DT)
    assert handed_to_collide(w) == 0 and w.stats()["rows"] == 590
    w.destroy()


def _rows_against_fresh(w):
    """Each row's deepest separation against a fresh collide() of its pair, and the tolerances."""
    w.begin_step(DT)
    copy = StageCopy(w)
    n = copy.count
    mem = _ffi.RowMemory()
    margin = np.zeros(max(n, 1))
    pid = np.zeros(P * max(n, 1), np.uint32)
    rem = np.zeros(max(n, 1), np.uint8)
    mpid = np.zeros(P * max(n, 1), np.uint32)
    memory = np.zeros(_ffi.BW_MEMORY * max(n, 1))
    mem.pid = pid.ctypes.data_as(C.POINTER(C.c_uint32))
    mem.margin = margin.ctypes.data_as(C.POINTER(C.c_double))
    mem.remembered = rem.ctypes.data_as(C.POINTER(C.c_uint8))
    mem.memory_pid = mpid.ctypes.data_as(C.POINTER(C.c_uint32))
    mem.memory = memory.ctypes.data_as(C.POINTER(C.c_double))
    assert w._lib.bw_row_memory_get(w._w, C.byref(mem)) == 0
    pairs = narrow_io.PairList(_ffi.Pairs(0))
    pairs.count = n
    pairs.a = copy.rows["a"][:n].astype(np.int32).copy()
    pairs.b = copy.rows["b"][:n].astype(np.int32).copy()
    pairs.margin = margin[:n].copy()
    pairs.tolerance = copy.rows["tolerance"][:n].copy()
    B, _, S = copy.views()
    fresh = narrow_io.host_collide(B, tuple(S.gravity), pairs)
    pts, got = copy.rows["points"].astype(np.int64), fresh.points.astype(np.int64)
    kept = np.array([copy.rows["separation"][P * m: P * m + pts[m]].min() for m in range(n)])
    found = np.array([fresh.separation[P * m: P * m + got[m]].min() if got[m] else np.inf for m in range(n)])
    w.end_step()
    return kept, found, pairs.tolerance


def test_a_kept_manifold_stays_within_the_tolerance_of_a_fresh_one():
    w = world(workers=4)
    scenes.pile(w, count=800, seed=11, extent=10.0)
    worst = 0.0
    checked = 0
    for i in range(90):
        w.step(DT)
        if i >= 40 and i % 10 == 0:
            kept, found, tol = _rows_against_fresh(w)
            # pairs in touch (REUSE's rules bound a touching pair's kept manifold; a pair apart but
            # within the margin, such as two boxes falling side by side, keeps the manifold it was
            # found with, which a fresh collide() with today's larger margin may place elsewhere)
            met = np.isfinite(found) & (found <= tol) & (kept <= tol)
            worst = max(worst, float(np.max(np.abs(kept[met] - found[met]) / tol[met])))
            checked += int(met.sum())
    assert checked > 300 and worst <= 1.0, worst
    w.destroy()


def test_fast_pairs_are_found_afresh_and_a_clone_keeps_the_cache():
    w = world()
    scenes.rain(w, count=300, seed=4)
    for _ in range(30):
        w.step(DT)
    w.begin_step(DT)
    assert handed_to_collide(w) > 0   # falling spheres' pairs move too fast to keep anything
    w.end_step()
    for _ in range(200):
        w.step(DT)
    clone = World({"reuse": True}, solver=oracle_io.solver(0))
    assert w._lib.bw_copy(clone._w, w._w) == 0
    clone._count = w._count
    for _ in range(20):
        w.step(DT)
        clone.step(DT)
    assert w.state()["position"].tobytes() == clone.state()["position"].tobytes()
    w.destroy()
    clone.destroy()


@pytest.mark.parametrize("reuse", [False, True])
def test_the_same_world_twice_to_the_bit(reuse):
    a, b = world(reuse), world(reuse)
    for w in (a, b):
        scenes.pile(w, count=300, seed=2, extent=6.0)
    for _ in range(60):
        a.step(DT)
        b.step(DT)
    assert a.state()["velocity"].tobytes() == b.state()["velocity"].tobytes()
    a.destroy()
    b.destroy()
