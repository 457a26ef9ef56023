"""Batched worlds on the GPU (one launch, one CTA a world) against the oracle, world by world."""
import numpy as np
import pytest

import oracle_io
from bearing_b200 import scenes
from bearing_b200.world import Batch, World

pytestmark = pytest.mark.gpu

DT = 1 / 60


def make(n, seed, solver):
    rng = np.random.default_rng(seed)
    worlds = []
    for _ in range(n):
        w = World({}, solver=solver)
        scenes.batch_world(w, rng)
        worlds.append(w)
    return worlds


def test_batched_worlds_match_the_oracle_world_by_world():
    gpu_worlds = make(48, 17, oracle_io.solver(0))
    ref_worlds = make(48, 17, oracle_io.solver(0))
    batch = Batch(gpu_worlds, threads=4)
    for step in range(40):
        batch.step(DT)
        for w in ref_worlds:
            w.step(DT)
    for i, (a, b) in enumerate(zip(gpu_worlds, ref_worlds)):
        sa, sb = a.state(), b.state()
        for k in sa:
            assert sa[k].tobytes() == sb[k].tobytes(), f"world {i}: {k}"
    assert sum(w.stats()["rows"] for w in gpu_worlds) > 1000
    batch.destroy()
