"""The oracle against its committed digests (tests/golden/oracle_digests.json, made by
tests/golden/make_oracle_digests.py): the pyramid and the 10-box stack, every step's FP64 body
state and contact columns, with the single-threaded solve and with worker threads (which must not
change a bit)."""
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_oracle_digests as golden  # noqa: E402

WANT = json.load(open(os.path.join(HERE, "golden", "oracle_digests.json")))


@pytest.mark.parametrize("scene", sorted(golden.SCENES))
@pytest.mark.parametrize("workers", [0, 3])
def test_oracle_matches_its_digests(scene, workers):
    got = golden.digests(scene, golden.SCENES[scene], workers)
    want = WANT[scene]
    for i, (g, w) in enumerate(zip(got, want)):
        assert g == w, f"{scene}, {workers} workers: step {i + 1} differs"
    assert len(got) == len(want)


def gpu_digests(scene, steps, flags):
    import hashlib
    from bearing_b200 import scenes
    from bearing_b200.world import GpuSolver, World
    solver = GpuSolver(0, flags)
    w = World({}, solver=solver)
    getattr(scenes, scene)(w)
    out = []
    for _ in range(steps):
        w.step(1 / 60)
        st, ct = w.state(), w.contacts()
        out.append(hashlib.sha256(b"".join(st[k].tobytes() for k in sorted(st))
                                  + b"".join(ct[k].tobytes() for k in sorted(ct))).hexdigest())
    w.destroy()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("scene", sorted(golden.SCENES))
@pytest.mark.parametrize("path", ["grid", "block"])
def test_gpu_matches_the_committed_digests(scene, path):
    from bearing_b200 import _ffi
    flags = _ffi.BG_FLAG_GRID if path == "grid" else _ffi.BG_FLAG_BLOCK
    got = gpu_digests(scene, golden.SCENES[scene], flags)
    for i, (g, w) in enumerate(zip(got, WANT[scene])):
        assert g == w, f"{scene} on the {path} path: step {i + 1} differs"
