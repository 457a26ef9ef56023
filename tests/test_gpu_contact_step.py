"""The whole contact side of a step on the device (bg_contact_step: the narrowphase, the rows and
their warm start from the contact memory, colouring and order, the solve stage, store and the
touching flags) against the host's rows stepped by the oracle's solve stage.

Two Worlds of the same scene: one steps on the host path with the oracle (its narrowphase, emit,
carry, colour, arrange, rest, keep and touched on the CPU), the other hands each step's pair list
to the device (World.set_contact_step) and gets back only the bodies.  Every body column the step
writes must be bit-identical after every checked step (NaN matching NaN), with the same row,
point, colour and overflow counts: any difference in a row, its warm start or its memory would
carry into the bodies within a step or two.
"""
import ctypes as C

import numpy as np
import pytest

import narrow_io
import oracle_io
from stage_io import StageCopy
from bearing_b200 import _ffi, scenes
from bearing_b200.world import GpuSolver, World

pytestmark = pytest.mark.gpu

DT = 1 / 60
REUSE = {"reuse": True}
_PI = C.POINTER(C.c_int32)
_PD = C.POINTER(C.c_double)


def _same(x, y):
    """Bit-identical arrays, a NaN matching any NaN (the CPU's and the GPU's NaN payloads differ)."""
    if x.dtype.kind == "f":
        both = np.isnan(x) & np.isnan(y)
        u = np.uint64 if x.dtype.itemsize == 8 else np.uint32
        return bool(np.all((x.view(u) == y.view(u)) | both))
    return x.tobytes() == y.tobytes()


def oracle_world(workers=0, options=None):
    return World(options or {}, solver=oracle_io.solver(workers))


def device_world(options=None):
    w = World(options or {})
    w.set_contact_step(w._solver)
    return w


def step_pair(build, steps, every=1, workers=0, options=None):
    """Steps both worlds `steps` times, comparing them at every `every`-th step and the last."""
    wa, wb = oracle_world(workers, options), device_world(options)
    build(wa)
    build(wb)
    most = 0
    for i in range(steps):
        wa.step(DT)
        wb.step(DT)
        if i % every == 0 or i == steps - 1:
            sa, sb = wa.state(), wb.state()
            for k in sa:
                assert _same(sa[k], sb[k]), f"step {i + 1}: {k} differs"
            ta, tb = wa.stats(), wb.stats()
            assert ta == tb, f"step {i + 1}: {ta} vs {tb}"
            assert _same(wa.transforms, wb.transforms), f"step {i + 1}: transforms differ"
            most = max(most, tb["rows"])
    ms = wb._contact.contact_ms()
    wa.destroy()
    wb.destroy()
    return most, ms


def test_pyramid_200_steps():
    most, ms = step_pair(scenes.pyramid, 200)
    assert most > 200 and ms is not None and all(t >= 0 for t in ms)


def test_overflow_slab():
    # A dynamic slab carrying 49 boxes: more rows on one body than there are colours.
    def build(w):
        scenes.ground(w)
        w.addBody({"size": (8.0, 0.5, 8.0), "position": (0.0, 0.25, 0.0), "density": 10.0})
        for i in range(7):
            for j in range(7):
                w.addBody({"size": (0.9, 0.9, 0.9), "position": (i - 3.0, 0.95, j - 3.0)})
    wb = device_world()
    build(wb)
    wb.step(DT)
    assert wb.stats()["overflow"] > 0
    wb.destroy()
    step_pair(build, 60)


def test_tumbling_boxes_and_capsules_with_restitution():
    def build(w):
        scenes.ground(w, friction=0.6)
        rng = np.random.default_rng(11)
        for i in range(40):
            q = rng.standard_normal(4)
            q = tuple(float(x) for x in q / np.linalg.norm(q))
            spin = tuple(float(x) for x in rng.uniform(-8, 8, 3))
            pos = (float(rng.uniform(-4, 4)), float(1 + 0.8 * i), float(rng.uniform(-4, 4)))
            if i % 2:
                w.addBody({"shape": "box", "size": tuple(float(x) for x in rng.uniform(0.3, 1.2, 3)), "rotation": q,
                           "position": pos, "angularVelocity": spin, "restitution": 0.2})
            else:
                r = float(rng.uniform(0.15, 0.3))
                w.addBody({"shape": "capsule", "radius": r, "height": 2 * (r + float(rng.uniform(0.2, 0.5))),
                           "rotation": q, "angularVelocity": spin, "position": pos, "friction": 0.3})
    step_pair(build, 180)


def test_kinematic_platform_and_spheres():
    # A kinematic platform sliding under boxes and spheres: rows with a kinematic side are coloured
    # on the dynamic body only, and emit()'s patch takes the dynamic body's size.
    def build(w):
        scenes.ground(w)
        w.addBody({"type": "kinematic", "size": (6.0, 0.4, 6.0), "position": (0.0, 1.0, 0.0),
                   "velocity": (0.5, 0.0, 0.0)})
        for i in range(5):
            for j in range(5):
                shape = {"shape": "sphere", "radius": 0.35} if (i + j) % 2 else {"size": (0.7, 0.7, 0.7)}
                w.addBody(dict(shape, position=(i - 2.0, 1.6 + 0.1 * j, j - 2.0), friction=0.4))
    step_pair(build, 90)


def test_rain_300_steps():
    # 2,000 spheres into a walled container with restitution; the state goes non-finite in the
    # reference's own arithmetic at step 172, and the two paths stay identical through it.
    most, _ = step_pair(lambda w: scenes.rain(w, count=2000, seed=2000), 300, every=10)
    assert most > 1000


def test_mixed_pile_3000():
    most, _ = step_pair(lambda w: scenes.pile(w, count=3000, seed=5, extent=30.0), 100, every=5)
    assert most > 2000


def test_the_50k_pile_120_steps():
    # The headline scene: 50,000 boxes, spheres and capsules landing in a pile, the oracle on 16
    # host threads on the other side.
    most, ms = step_pair(lambda w: scenes.pile(w, count=50_000, seed=50_000), 120, every=20, workers=16)
    assert most > 60_000 and ms is not None


def test_bodies_added_between_steps():
    # The World's columns grow under the contact step (new slots, new pairs, the pair list's slots
    # moving), and its records still follow their pairs.
    wa, wb = oracle_world(options=REUSE), device_world(REUSE)
    for w in (wa, wb):
        scenes.pyramid(w, rows=8)
    rng = np.random.default_rng(3)
    drops = [(float(rng.uniform(-2, 2)), float(6 + i), float(rng.uniform(-2, 2))) for i in range(12)]
    for i in range(150):
        if i in (30, 60, 90):
            for w in (wa, wb):
                for p in drops[(i // 30 - 1) * 4:(i // 30) * 4]:
                    shape = {"shape": "sphere", "radius": 0.3} if p[1] % 2 else {"size": (0.6, 0.6, 0.6)}
                    w.addBody(dict(shape, position=p))
        wa.step(DT)
        wb.step(DT)
        sa, sb = wa.state(), wb.state()
        for k in sa:
            assert _same(sa[k], sb[k]), f"step {i + 1}: {k} differs"
        assert wa.stats() == wb.stats(), f"step {i + 1}"
    wa.destroy()
    wb.destroy()


# ---- with the kept-manifold cache (src/contact.js:388-595), kept in the device's records ----

def test_pyramid_reusing_kept_manifolds():
    most, _ = step_pair(scenes.pyramid, 200, options=REUSE)
    assert most > 200


def test_tumbling_and_kinematic_reusing_kept_manifolds():
    def build(w):
        scenes.ground(w, friction=0.6)
        w.addBody({"type": "kinematic", "size": (6.0, 0.4, 6.0), "position": (0.0, 1.0, 0.0),
                   "velocity": (0.3, 0.0, 0.0), "angularVelocity": (0.0, 0.4, 0.0)})
        rng = np.random.default_rng(5)
        for i in range(30):
            q = rng.standard_normal(4)
            q = tuple(float(x) for x in q / np.linalg.norm(q))
            pos = (float(rng.uniform(-2.5, 2.5)), float(1.8 + 0.6 * i), float(rng.uniform(-2.5, 2.5)))
            if i % 3 == 0:
                w.addBody({"shape": "capsule", "radius": 0.2, "height": 0.9, "rotation": q, "position": pos})
            elif i % 3 == 1:
                w.addBody({"shape": "sphere", "radius": 0.3, "position": pos, "restitution": 0.3})
            else:
                w.addBody({"size": (0.6, 0.4, 0.5), "rotation": q, "position": pos})
    step_pair(build, 150, options=REUSE)


def test_rain_reusing_kept_manifolds():
    most, _ = step_pair(lambda w: scenes.rain(w, count=2000, seed=2000), 300, every=10, options=REUSE)
    assert most > 1000


def test_mixed_pile_3000_reusing_kept_manifolds():
    most, _ = step_pair(lambda w: scenes.pile(w, count=3000, seed=5, extent=30.0), 100, every=5, options=REUSE)
    assert most > 2000


def test_the_50k_pile_reusing_kept_manifolds():
    most, _ = step_pair(lambda w: scenes.pile(w, count=50_000, seed=50_000), 120, every=20, workers=16,
                        options=REUSE)
    assert most > 60_000


# ---- the C ABI directly ----

def _inputs(steps=10):
    """A pyramid's bodies after `steps` steps, its pair list, and materials, as the host hands them."""
    w = oracle_world()
    scenes.pyramid(w, rows=6)
    for _ in range(steps):
        w.step(DT)
    w.begin_step(DT)
    copy = StageCopy(w)
    pairs = narrow_io.world_pairs(w)
    n = copy.capacity
    fr = np.empty(n)
    rs = np.empty(n)
    assert w._lib.bw_materials(w._w, fr.ctypes.data_as(_PD), rs.ctypes.data_as(_PD)) == 0
    w.destroy()
    return copy, pairs, fr, rs


def _call(lib, ctx, copy, pairs, fr, rs, memory):
    B, _, S = copy.views()
    size = np.ones(copy.capacity)
    M = _ffi.Materials(fr.ctypes.data_as(_PD), rs.ctypes.data_as(_PD), size.ctypes.data_as(_PD))
    mem = np.ascontiguousarray(memory, np.int32)
    CP = _ffi.ContactPairs(pairs.view(), mem.ctypes.data_as(_PI))
    n = max(pairs.count, 1)
    pts, tch = np.full(n, 0xAB, np.uint8), np.full(n, 0xAB, np.uint8)
    out = _ffi.ContactResult()
    out.points = pts.ctypes.data_as(C.POINTER(C.c_uint8))
    out.touching = tch.ctypes.data_as(C.POINTER(C.c_uint8))
    rc = lib.bg_contact_step(ctx, C.byref(B), C.byref(M), C.byref(CP), C.byref(S), C.byref(out))
    return rc, pts[: pairs.count], tch[: pairs.count], out


def test_point_counts_are_the_host_narrowphase_and_refusals_write_nothing():
    copy, pairs, fr, rs = _inputs()
    B, _, S = copy.views()
    want = narrow_io.host_collide(B, S.gravity, pairs)
    s = GpuSolver()
    lib = s.lib
    none = -np.ones(pairs.count, np.int32)
    # refused before anything is copied: the bodies stay as they were, no records are made
    before = {k: v.copy() for k, v in copy.body.items()}
    bad_slot = narrow_io.PairList(pairs.view())
    bad_slot.b[3] = copy.capacity
    same_slot = narrow_io.PairList(pairs.view())
    same_slot.b[1] = same_slot.a[1]
    for p, mem in ((bad_slot, none), (same_slot, none), (pairs, np.where(np.arange(pairs.count) == 2, 0, -1))):
        rc, _, _, _ = _call(lib, s.ctx, copy, p, fr, rs, mem)
        assert rc == _ffi.BG_EINVAL, s.error()
        assert all(before[k].tobytes() == copy.body[k].tobytes() for k in before)
        assert lib.bg_contact_records(s.ctx) == 0
    rc, pts, tch, out = _call(lib, s.ctx, copy, pairs, fr, rs, none)
    assert rc == 0, s.error()
    assert np.array_equal(pts, want.points[: pairs.count])
    assert out.rows == int(np.count_nonzero(pts)) and out.solved <= out.rows
    assert set(np.unique(tch)) <= {0, 1} and not np.any(tch[pts == 0])
    assert lib.bg_contact_records(s.ctx) == pairs.count
    # a record past the last list is refused; forgetting clears them
    mem = np.where(np.arange(pairs.count) == 0, pairs.count, -1)
    assert _call(lib, s.ctx, copy, pairs, fr, rs, mem)[0] == _ffi.BG_EINVAL
    assert lib.bg_contact_forget(s.ctx) == 0 and lib.bg_contact_records(s.ctx) == 0
    s.close()


def test_an_empty_list_still_steps_the_bodies():
    w = device_world()
    w.addBody({"position": (0.0, 5.0, 0.0), "velocity": (1.0, 0.0, 0.0)})
    wa = oracle_world()
    wa.addBody({"position": (0.0, 5.0, 0.0), "velocity": (1.0, 0.0, 0.0)})
    for _ in range(5):
        w.step(DT)
        wa.step(DT)
    sa, sb = wa.state(), w.state()
    assert all(_same(sa[k], sb[k]) for k in sa)
    assert w.stats()["rows"] == 0
    w.destroy()
    wa.destroy()


def test_a_lost_contact_step_keeps_the_records_and_the_retry_matches():
    # A wait budget of one iteration makes the colouring's waits run out: the call returns
    # BG_ETIMEOUT (the reference's Jobs.lost), holds no new records, and the same call with the
    # default budget then gives exactly what a context that never lost the step gives.
    w = oracle_world()
    scenes.pile(w, count=2000, seed=9, extent=14.0)
    for _ in range(60):
        w.step(DT)
    w.begin_step(DT)
    copy = StageCopy(w)
    pairs = narrow_io.world_pairs(w)
    fr, rs = np.empty(copy.capacity), np.empty(copy.capacity)
    assert w._lib.bw_materials(w._w, fr.ctypes.data_as(_PD), rs.ctypes.data_as(_PD)) == 0
    w.destroy()
    none = -np.ones(pairs.count, np.int32)
    good, lost = GpuSolver(), GpuSolver()
    want = copy.copy()
    rc, _, _, out = _call(good.lib, good.ctx, want, pairs, fr, rs, none)
    assert rc == 0 and out.rows > 1000
    got = copy.copy()
    assert lost.lib.bg_set_wait_budget(lost.ctx, 1) == 0
    rc, _, _, _ = _call(lost.lib, lost.ctx, got, pairs, fr, rs, none)
    assert rc == _ffi.BG_ETIMEOUT, lost.error()
    assert lost.lib.bg_contact_records(lost.ctx) == 0
    assert lost.lib.bg_set_wait_budget(lost.ctx, 1 << 24) == 0
    got = copy.copy()
    rc, _, _, _ = _call(lost.lib, lost.ctx, got, pairs, fr, rs, none)
    assert rc == 0, lost.error()
    for f in got.body:
        assert _same(got.body[f], want.body[f]), f
    assert lost.lib.bg_contact_records(lost.ctx) == pairs.count
    good.close()
    lost.close()
