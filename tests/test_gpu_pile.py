"""The headline workload end to end: the 50,000-body mixed pile stepped 300 times by a World whose
solve stage runs on the GPU, and by the same World on the oracle (every host thread), compared by
a digest of every FP64 body column the stage writes and the step's contact columns every 50 steps
(the pile lands, peaks at ~145k rows near step 100 and settles to ~123k by step 300).  About two
minutes on one B200 and its host."""
import hashlib
import os

import pytest

import oracle_io
from bearing_b200 import scenes
from bearing_b200.world import GpuSolver, World

pytestmark = pytest.mark.gpu


def digest(w):
    """Every FP64 body column the stage writes, and the last step's contact columns."""
    st, ct = w.state(), w.contacts()
    return hashlib.sha256(b"".join(st[k].tobytes() for k in sorted(st))
                          + b"".join(ct[k].tobytes() for k in sorted(ct))).hexdigest()


def test_pile_of_50k_bodies_300_steps_bit_identical_to_the_oracle():
    threads = len(os.sched_getaffinity(0))
    gpu = World({}, solver=GpuSolver())
    ref = World({}, solver=oracle_io.solver(max(0, threads - 1)))
    for w in (gpu, ref):
        scenes.pile(w, count=50_000, seed=50_000)
    try:
        for i in range(300):
            gpu.step(1 / 60)
            ref.step(1 / 60)
            if (i + 1) % 50 == 0:
                assert digest(gpu) == digest(ref), f"step {i + 1}"
        assert gpu.stats()["rows"] > 100_000
    finally:
        gpu.destroy()
        ref.destroy()
