"""The benchmark scenes, as seeded synthetic worlds.

Each builder adds bodies to a World (or anything with ``addBody(spec)``) and returns the slots
it added.  The shapes, sizes and value distributions are the ones the benchmark configurations
name; every random draw comes from numpy's PCG64 with the seed given.

  pyramid   20 rows, row k of 20-k unit cubes at [j - (19-k)/2, 0.5 + k, 0] on a static
            100 x 1 x 100 ground (test/contact.test.js:45-64, bench/solver.js:78-84);
            friction 0.6 for the pyramid config.
  stack     ten unit cubes one on another (test/contact.test.js:30-43).
  rain      2,000 spheres, r ~ U(0.25, 0.5), friction 0.5, restitution 0.3, dropped from a
            10 x 40 x 10 m volume into a walled container (floor 12 x 1 x 12, four 1 x 12 x 12
            walls; the two z-walls are 12 x 12 x 1).
  pile      50,000 mixed bodies: 60% boxes (half-extents U(0.2, 0.6)), 25% spheres
            (r U(0.2, 0.5)), 15% capsules (r U(0.15, 0.3), half-height U(0.2, 0.5), so
            height = 2 (hh + r)); normalised-Gaussian orientations; a 1.5 m grid jittered
            +-0.2 m; friction 0.6, restitution 0.1; dropped on a walled 100 x 1 x 100 ground.
  batch     worlds of log-uniform 8..512 bodies, each a pyramid, a box stack or a sphere
            pile, friction U(0.3, 0.8), restitution U(0, 0.4).
  tower     a 3 x 10 tower of 0.5 m cubes struck by a 0.5 m, 50 kg sphere at 5..15 m/s, with
            friction U(0.2, 0.9) and restitution U(0, 0.5) for every body; the loss is the
            squared distance of the cubes' final centres from seeded targets.
"""
from __future__ import annotations

import math

import numpy as np


def ground(world, size=(100.0, 1.0, 100.0), friction=0.5, y=-0.5):
    return world.addBody({"type": "static", "size": size, "position": (0.0, y, 0.0), "friction": friction})


def pyramid(world, rows=20, friction=0.6, ground_friction=0.6):
    """The 210-box pyramid: ground at y = -0.5, then rows of unit cubes."""
    slots = [ground(world, friction=ground_friction)]
    for row in range(rows):
        for k in range(rows - row):
            at = (k - (rows - 1 - row) / 2, 0.5 + row, 0.0)
            slots.append(world.addBody({"position": at, "friction": friction}))
    return slots


def stack(world, count=10, friction=0.5):
    slots = [ground(world, friction=friction)]
    for k in range(count):
        slots.append(world.addBody({"position": (0.0, 0.5 + k, 0.0), "friction": friction}))
    return slots


def container(world, half=6.0, wall=12.0, friction=0.5):
    """A static floor (2half x 1 x 2half) and four walls around it."""
    slots = [world.addBody({"type": "static", "size": (2 * half, 1.0, 2 * half), "position": (0.0, -0.5, 0.0),
                            "friction": friction})]
    h = wall / 2
    for sx in (-1, 1):
        slots.append(world.addBody({"type": "static", "size": (1.0, wall, wall),
                                    "position": (sx * (half + 0.5), h - 1.0, 0.0), "friction": friction}))
    for sz in (-1, 1):
        slots.append(world.addBody({"type": "static", "size": (wall, wall, 1.0),
                                    "position": (0.0, h - 1.0, sz * (half + 0.5)), "friction": friction}))
    return slots


def rain(world, count=2000, seed=2000):
    """2,000 spheres raining into a walled container."""
    rng = np.random.default_rng(seed)
    slots = container(world, friction=0.5)
    r = rng.uniform(0.25, 0.5, count)
    xs = rng.uniform(-5.0, 5.0, count)
    ys = rng.uniform(2.0, 42.0, count)
    zs = rng.uniform(-5.0, 5.0, count)
    for i in range(count):
        slots.append(world.addBody({"shape": "sphere", "radius": float(r[i]), "friction": 0.5, "restitution": 0.3,
                                    "position": (float(xs[i]), float(ys[i]), float(zs[i]))}))
    return slots


def _gauss_quat(rng):
    q = rng.standard_normal(4)
    return tuple(float(x) for x in q / np.linalg.norm(q))


def pile(world, count=50_000, seed=50_000, spacing=1.5, jitter=0.2, extent=100.0):
    """The 50k-body mixed pile on a walled ground."""
    rng = np.random.default_rng(seed)
    half = extent / 2
    slots = [world.addBody({"type": "static", "size": (extent, 1.0, extent), "position": (0.0, -0.5, 0.0),
                            "friction": 0.6, "restitution": 0.1})]
    wall = 8.0
    for sx in (-1, 1):
        slots.append(world.addBody({"type": "static", "size": (1.0, wall, extent),
                                    "position": (sx * (half + 0.5), wall / 2 - 1.0, 0.0), "friction": 0.6,
                                    "restitution": 0.1}))
    for sz in (-1, 1):
        slots.append(world.addBody({"type": "static", "size": (extent, wall, 1.0),
                                    "position": (0.0, wall / 2 - 1.0, sz * (half + 0.5)), "friction": 0.6,
                                    "restitution": 0.1}))
    per_side = int((extent - 2 * spacing) // spacing)
    per_layer = per_side * per_side
    kinds = rng.permutation(np.array([0] * int(count * 0.60) + [1] * int(count * 0.25)
                                     + [2] * (count - int(count * 0.60) - int(count * 0.25))))
    for i in range(count):
        layer, k = divmod(i, per_layer)
        gx, gz = divmod(k, per_side)
        x = -half + spacing * (gx + 1) + rng.uniform(-jitter, jitter)
        z = -half + spacing * (gz + 1) + rng.uniform(-jitter, jitter)
        y = 1.0 + spacing * layer + rng.uniform(-jitter, jitter)
        q = _gauss_quat(rng)
        spec = {"position": (x, y, z), "rotation": q, "friction": 0.6, "restitution": 0.1}
        if kinds[i] == 0:
            h = rng.uniform(0.2, 0.6, 3)
            spec.update(shape="box", size=tuple(float(2 * v) for v in h))
        elif kinds[i] == 1:
            spec.update(shape="sphere", radius=float(rng.uniform(0.2, 0.5)))
        else:
            r = float(rng.uniform(0.15, 0.3))
            hh = float(rng.uniform(0.2, 0.5))
            spec.update(shape="capsule", radius=r, height=2 * (hh + r))
        slots.append(world.addBody(spec))
    return slots


def batch_rng(seed, i):
    """World i's own generator in a batch: worlds draw independently, so any subset of a batch
    (one rank's shard) builds exactly as it would in the whole batch."""
    return np.random.default_rng([seed, i])


def batch_world_bodies(rng_seed, i):
    """The body count batch_world draws first for world i (its weight when sharding)."""
    rng = batch_rng(rng_seed, i)
    return int(round(math.exp(rng.uniform(math.log(8), math.log(512)))))


def batch_world(world, rng):
    """One world of the batch: a pyramid, a box stack or a sphere pile of 8..512 bodies."""
    n = int(round(math.exp(rng.uniform(math.log(8), math.log(512)))))
    mu = float(rng.uniform(0.3, 0.8))
    e = float(rng.uniform(0.0, 0.4))
    kind = int(rng.integers(0, 3))
    slots = [world.addBody({"type": "static", "size": (40.0, 1.0, 40.0), "position": (0.0, -0.5, 0.0),
                            "friction": mu, "restitution": e})]
    if kind == 0:
        rows = 1
        while rows * (rows + 1) // 2 < n:
            rows += 1
        placed = 0
        for row in range(rows):
            for k in range(rows - row):
                if placed == n:
                    break
                slots.append(world.addBody({"position": (k - (rows - 1 - row) / 2, 0.5 + row, 0.0),
                                            "friction": mu, "restitution": e}))
                placed += 1
    elif kind == 1:
        side = max(1, int(round(n ** (1 / 3))))
        for i in range(n):
            layer, k = divmod(i, side * side)
            gx, gz = divmod(k, side)
            slots.append(world.addBody({"position": (1.05 * gx - side / 2, 0.5 + layer, 1.05 * gz - side / 2),
                                        "friction": mu, "restitution": e}))
    else:
        side = max(1, int(math.ceil(math.sqrt(n / 4))))
        for i in range(n):
            layer, k = divmod(i, side * side)
            gx, gz = divmod(k, side)
            r = float(rng.uniform(0.25, 0.5))
            slots.append(world.addBody({"shape": "sphere", "radius": r, "friction": mu, "restitution": e,
                                        "position": (1.1 * gx - side / 2 + rng.uniform(-0.05, 0.05),
                                                     0.6 + 1.1 * layer, 1.1 * gz - side / 2)}))
    return kind, slots


def tower_targets(rng, centres):
    """The loss's targets for the tower's cubes: each cube's starting centre moved by N(0, 0.1) m
    on every axis, drawn after the scene's own draws."""
    centres = np.asarray(centres, dtype=np.float64)
    return centres + rng.normal(0.0, 0.1, centres.shape)


def tower(world, rng):
    """The differentiable scene: a 3 x 10 tower of 0.5 m cubes and a 50 kg ball thrown at it.
    Returns the slots and the draws: friction, restitution, speed, the cubes' and the ball's slots,
    and the loss's targets for the cubes (tower_targets)."""
    mu = float(rng.uniform(0.2, 0.9))
    e = float(rng.uniform(0.0, 0.5))
    speed = float(rng.uniform(5.0, 15.0))
    slots = [world.addBody({"type": "static", "size": (40.0, 1.0, 40.0), "position": (0.0, -0.5, 0.0),
                            "friction": mu, "restitution": e})]
    cubes, centres = [], []
    for layer in range(10):
        for k in range(3):
            centres.append((0.5 * k - 0.5, 0.25 + 0.5 * layer, 0.0))
            cubes.append(world.addBody({"size": (0.5, 0.5, 0.5), "position": centres[-1],
                                        "friction": mu, "restitution": e}))
    ball = world.addBody({"shape": "sphere", "radius": 0.5, "mass": 50.0, "friction": mu, "restitution": e,
                          "position": (-0.5, 0.5, -4.0), "velocity": (0.0, 0.0, speed)})
    return slots + cubes + [ball], dict(friction=mu, restitution=e, speed=speed, cubes=cubes, ball=ball,
                                        targets=tower_targets(rng, centres))


def tower_loss(position, info, body0=0):
    """The tower's loss, the sum over its cubes of the squared distance from each cube's centre to
    its target, and the loss's adjoint of every position (3 per slot, from slot body0)."""
    cubes = np.asarray(info["cubes"], dtype=np.int64) + body0
    idx = (3 * cubes[:, None] + np.arange(3)[None, :])
    d = position[idx] - info["targets"]
    seed = np.zeros_like(position)
    seed[idx] = 2 * d
    return float(np.sum(d * d)), seed

