"""The CUDA solve stage against the oracle, bit for bit.

Each case runs the host side of a step (``World.begin_step``), copies the solve stage's input,
runs it once through the oracle and once through ``bg_solve_step`` and requires every column the
stage writes to be bit-identical.  The multi-step cases step two worlds, one with each solver,
and require identical FP64 state throughout: any difference in any step would carry on.
"""
import numpy as np
import pytest

import gpu_io
import oracle_io
from stage_io import BODY_COLUMNS, ROW_COLUMNS, StageCopy, first_difference
from bearing_b200 import scenes
from bearing_b200.world import World

pytestmark = pytest.mark.gpu

DT = 1 / 60


def oracle_world(options=None):
    return World(options or {}, solver=oracle_io.solver(0))


def gpu_world(options=None):
    return World(options or {})


def finish_with(world, copy):
    """Writes copy's solved columns back into the world and ends its step."""
    B, R, _ = world.views()
    for f, dt, per in BODY_COLUMNS:
        n = per * copy.capacity
        if n:
            np.ctypeslib.as_array(getattr(B, f), shape=(n,))[:] = copy.body[f]
    for f, dt, per in ROW_COLUMNS:
        n = per * copy.count
        if n:
            np.ctypeslib.as_array(getattr(R, f), shape=(n,))[:] = copy.rows[f]
    world.end_step()


def run_pair(build, steps, check_every=1):
    """Steps a world `steps` times; at each checked step the GPU and the oracle solve the same
    input.  Returns the number of rows seen."""
    w = oracle_world()
    build(w)
    rows = 0
    for i in range(steps):
        w.begin_step(DT)
        base = StageCopy(w)
        a = oracle_io.solve(base.copy())
        if i % check_every == 0 or i == steps - 1:
            b = gpu_io.solve(base.copy())
            diff = first_difference(a, b)
            assert diff is None, f"step {i + 1}: {diff}"
            rows = max(rows, base.count)
        finish_with(w, a)
    return rows


def test_pyramid_first_step():
    w = oracle_world()
    scenes.pyramid(w)
    w.begin_step(DT)
    base = StageCopy(w)
    assert base.count > 400
    a = oracle_io.solve(base.copy())
    b = gpu_io.solve(base.copy())
    assert first_difference(a, b) is None


def test_pyramid_every_step_for_120_steps():
    assert run_pair(scenes.pyramid, 120) > 400


def test_stack_every_step():
    run_pair(scenes.stack, 60)


def test_spheres_bouncing_restitution():
    # bouncy spheres exercise restitution(), the rolling and spin rows, and 1-point manifolds
    def build(w):
        scenes.ground(w)
        rng = np.random.default_rng(7)
        for i in range(60):
            w.addBody({"shape": "sphere", "radius": float(rng.uniform(0.2, 0.5)), "restitution": 0.7,
                       "position": (float(rng.uniform(-3, 3)), float(rng.uniform(0.6, 6)), float(rng.uniform(-3, 3))),
                       "angularVelocity": (0.0, float(rng.uniform(-5, 5)), 0.0)})
    run_pair(build, 200)


def test_mixed_shapes_tumbling():
    # lopsided boxes and capsules, spinning: tumble() and untwist() on the device
    def build(w):
        scenes.ground(w, friction=0.6)
        rng = np.random.default_rng(11)
        for i in range(40):
            q = rng.standard_normal(4)
            q = tuple(float(x) for x in q / np.linalg.norm(q))
            spin = tuple(float(x) for x in rng.uniform(-8, 8, 3))
            if i % 2:
                w.addBody({"shape": "box", "size": tuple(float(x) for x in rng.uniform(0.3, 1.2, 3)), "rotation": q,
                           "position": (float(rng.uniform(-4, 4)), float(1 + 0.8 * i), float(rng.uniform(-4, 4))),
                           "angularVelocity": spin, "restitution": 0.2})
            else:
                r = float(rng.uniform(0.15, 0.3))
                w.addBody({"shape": "capsule", "radius": r, "height": 2 * (r + float(rng.uniform(0.2, 0.5))),
                           "rotation": q, "angularVelocity": spin,
                           "position": (float(rng.uniform(-4, 4)), float(1 + 0.8 * i), float(rng.uniform(-4, 4)))})
    run_pair(build, 180)


def test_overflow_colour():
    # A dynamic slab carrying 49 boxes: its rows use every colour and the rest overflow
    # (test/contact.test.js:186-216); the overflow is solved in row order.
    def build(w):
        scenes.ground(w)
        w.addBody({"size": (8.0, 0.5, 8.0), "position": (0.0, 0.25, 0.0), "density": 10.0})
        for i in range(7):
            for j in range(7):
                w.addBody({"size": (0.9, 0.9, 0.9), "position": (i - 3.0, 0.95, j - 3.0)})
    w = oracle_world()
    build(w)
    w.begin_step(DT)
    base = StageCopy(w)
    assert base.starts[33] > base.starts[32], "expected rows in the overflow colour"
    a = oracle_io.solve(base.copy())
    for path in ("grid", "block"):   # the grid takes the overflow one row a run, in rank order
        b = gpu_io.solve(base.copy(), path)
        assert first_difference(a, b) is None, path
    finish_with(w, a)
    for i in range(20):
        w.begin_step(DT)
        base = StageCopy(w)
        a = oracle_io.solve(base.copy())
        b = gpu_io.solve(base.copy(), "grid")
        assert first_difference(a, b) is None, f"grid, step {i + 2}"
        finish_with(w, a)
    assert run_pair(build, 30) > 0


def test_locked_and_frozen_bodies():
    # lockedInverse() and frozen bodies, set on a copy of a real step's input
    w = oracle_world()
    scenes.pyramid(w, rows=8)
    for _ in range(5):
        w.step(DT)
    w.begin_step(DT)
    base = StageCopy(w)
    slots = base.awake_list
    base.body["lock"][slots[::3]] = 1
    base.body["lock"][slots[1::5]] = 5
    base.body["lock"][slots[2::7]] = 7
    frozen = slots[4::6]
    base.body["frozen"][frozen] = 1
    base.body["inv_mass"][frozen] = 0.0
    a = oracle_io.solve(base.copy())
    b = gpu_io.solve(base.copy())
    assert first_difference(a, b) is None


@pytest.mark.parametrize("path", ["grid", "block"])
def test_awake_bodies_without_mass_and_moved_bodies_not_awake(path):
    # Two inputs the grid's body passes treat apart, on both paths: awake bodies with inverse mass
    # 0 (frozen here; kinematic alike), whose moves no counter orders, so the move pass keeps its
    # grid barriers; and dynamic bodies the rows move that are not on the awake list, which are
    # neither accelerated nor moved but still take their turns.
    w = oracle_world()
    scenes.pyramid(w)
    for _ in range(4):
        w.step(DT)
    w.begin_step(DT)
    base = StageCopy(w)
    slots = base.awake_list.copy()
    frozen = slots[5::9]
    base.body["frozen"][frozen] = 1
    base.body["inv_mass"][frozen] = 0.0
    a = oracle_io.solve(base.copy())
    b = gpu_io.solve(base.copy(), path)
    assert first_difference(a, b) is None, "frozen awake bodies"
    base = StageCopy(w)
    dropped = set(int(x) for x in slots[3::7])
    kept = np.array([x for x in slots if int(x) not in dropped], dtype=np.int32)
    base.awake_list = kept
    base.awake_count = len(kept)
    for x in dropped:
        base.body["awake"][x] = 0
    a = oracle_io.solve(base.copy())
    b = gpu_io.solve(base.copy(), path)
    assert first_difference(a, b) is None, "moved bodies off the awake list"


def test_no_contacts_free_fall():
    w = oracle_world()
    w.addBody({"position": (0.0, 10.0, 0.0), "angularVelocity": (1.0, 2.0, 3.0), "size": (1.0, 2.0, 3.0)})
    w.begin_step(DT)
    base = StageCopy(w)
    assert base.count == 0
    a = oracle_io.solve(base.copy())
    b = gpu_io.solve(base.copy())
    assert first_difference(a, b) is None


@pytest.mark.parametrize("path", ["grid", "block"])
def test_both_paths_on_a_mixed_pile(path):
    # The persistent grid (large worlds) and the one-CTA path (small and batched worlds) on the
    # same inputs, a landing pile of boxes, spheres and capsules with restitution.
    def build(w):
        scenes.pile(w, count=3000, seed=5, extent=30.0)
    w = oracle_world()
    build(w)
    for i in range(40):
        w.step(DT)
    for i in range(3):
        w.begin_step(DT)
        base = StageCopy(w)
        assert base.solved > 1000
        a = oracle_io.solve(base.copy())
        b = gpu_io.solve(base.copy(), path)
        assert first_difference(a, b) is None, f"step {41 + i}"
        finish_with(w, a)


def test_pyramid_on_the_grid_path():
    w = oracle_world()
    scenes.pyramid(w)
    for i in range(30):
        w.begin_step(DT)
        base = StageCopy(w)
        a = oracle_io.solve(base.copy())
        b = gpu_io.solve(base.copy(), "grid")
        assert first_difference(a, b) is None, f"step {i + 1}"
        finish_with(w, a)


def _same(x, y):
    """Bit-identical arrays, a NaN matching any NaN (the CPU's and the GPU's NaN payloads differ)."""
    if x.dtype.kind == "f":
        both = np.isnan(x) & np.isnan(y)
        u = np.uint64 if x.dtype == np.float64 else np.uint32
        return bool(np.all((x.view(u) == y.view(u)) | both))
    return x.tobytes() == y.tobytes()


@pytest.mark.parametrize("config", ["pyramid", "rain"])
def test_gpu_world_matches_oracle_world_over_600_steps(config):
    # The whole loop on the two parity workloads: the 20-row pyramid (210 boxes) and 2,000
    # spheres raining into a walled container, 600 steps each, a World on the GPU against the
    # same World on the oracle, state and transforms identical after every step.  The rain goes
    # non-finite in the reference's own arithmetic at step 172 (a contact's normal impulse has
    # decayed to 3.3e-163, the friction limit's square underflows to 0 and the cone's Newton
    # step overflows); restitution's push() then writes the NaN into a static wall and on in
    # found order, and the GPU follows it there too, so the two stay identical (NaN matching
    # NaN) through all 600 steps.
    wa, wb = oracle_world(), gpu_world()
    for w in (wa, wb):
        if config == "pyramid":
            scenes.pyramid(w)
        else:
            scenes.rain(w, count=2000, seed=2000)
    first_nonfinite = None
    for i in range(600):
        wa.step(DT)
        wb.step(DT)
        sa, sb = wa.state(), wb.state()
        motion = ("position", "rotation", "velocity", "angular")   # ceiling starts at +inf
        if first_nonfinite is None and not all(np.all(np.isfinite(sa[k])) for k in motion):
            first_nonfinite = i + 1
        for k in sa:
            assert _same(sa[k], sb[k]), f"step {i + 1}: {k}"
        assert _same(wa.transforms, wb.transforms), f"step {i + 1}: transforms"
    assert first_nonfinite == (None if config == "pyramid" else 172), first_nonfinite
    assert wa.stats()["rows"] > 100 or config == "rain"
