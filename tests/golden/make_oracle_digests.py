"""Writes oracle_digests.json: per-step SHA-256 digests of the oracle's full FP64 body state and
contact columns for two of the reference's own test scenes, stepped through the host side of the
step and the oracle's solve stage (tests/test_golden.py checks them).

The reference stores no numeric vectors of its own (its tests check behaviour with tolerances),
so these pin this repository's CPU restatement against unintended change, not against the
reference; regenerate them only for a deliberate change of the oracle:

    python tests/golden/make_oracle_digests.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

SCENES = {"pyramid": 40, "stack": 40}   # scene -> steps at 1/60 s


def digests(scene, steps, workers=0):
    import oracle_io
    from bearing_b200 import scenes
    from bearing_b200.world import World
    w = World({}, solver=oracle_io.solver(workers))
    getattr(scenes, scene)(w)
    out = []
    for _ in range(steps):
        w.step(1 / 60)
        st, ct = w.state(), w.contacts()
        out.append(hashlib.sha256(b"".join(st[k].tobytes() for k in sorted(st))
                                  + b"".join(ct[k].tobytes() for k in sorted(ct))).hexdigest())
    w.destroy()
    return out


if __name__ == "__main__":
    data = {name: digests(name, steps) for name, steps in SCENES.items()}
    with open(os.path.join(HERE, "oracle_digests.json"), "w") as f:
        json.dump(data, f, indent=1)
        f.write("\n")
    print({k: len(v) for k, v in data.items()})
