"""The host's share of a step whose contact side runs on another device (bw_set_contact_step): the
pair list's upkeep (src/pairs.js found/remove/forget) and each pair's contact record, checked with a
stand-in for the device that remembers every list it was handed.  No GPU: the stand-in decides which
pairs touch and moves bodies away so that pairs are removed and the pair list's slots move."""
import ctypes as C

import pytest

import oracle_io
from bearing_b200 import _ffi, scenes
from bearing_b200.world import BearingError, World

DT = 1 / 60
PROTO = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.POINTER(_ffi.Bodies), C.POINTER(_ffi.Materials),
                    C.POINTER(_ffi.ContactPairs), C.POINTER(_ffi.Step), C.POINTER(_ffi.ContactResult))


class StandIn:
    """Answers each call as a device would, and checks each pair's record against the last list:
    a record names the same pair, which touched; a pair that touched last time and is listed again
    names its record."""

    def __init__(self, move_on=2, moved=12):
        self.prev = []          # ((a, b), touched) of the last list, by index
        self.problems = []
        self.calls = 0
        self.carried = 0        # pairs that named a record
        self.move_on, self.moved = move_on, moved
        self.last = None
        self.fn = PROTO(self)

    def touches(self, a, b):
        return (a * 31 + b * 17 + self.calls) % 5 != 0

    def __call__(self, user, bodies, materials, pairs, step, out):
        try:
            cp, B = pairs.contents, bodies.contents
            n = cp.list.count
            ab = [(cp.list.a[i], cp.list.b[i]) for i in range(n)]
            mem = [cp.memory[i] for i in range(n)]
            touched_before = {k for k, t in self.prev if t}
            for i, (key, j) in enumerate(zip(ab, mem)):
                if j >= 0:
                    self.carried += 1
                    if j >= len(self.prev) or self.prev[j][0] != key or not self.prev[j][1]:
                        self.problems.append(f"call {self.calls}: pair {key} names record {j}")
                elif key in touched_before:
                    self.problems.append(f"call {self.calls}: pair {key} touched last step but names no record")
                if not (0 <= key[0] < B.capacity and 0 <= key[1] < B.capacity) or key[0] >= key[1]:
                    self.problems.append(f"call {self.calls}: pair {key} out of order or range")
                if not (cp.list.margin[i] >= cp.list.tolerance[i] > 0):
                    self.problems.append(f"call {self.calls}: pair {key} margin {cp.list.margin[i]}")
            touch = [self.touches(a, b) for a, b in ab]
            for i, t in enumerate(touch):
                out.contents.points[i] = 2 if t else 0
                out.contents.touching[i] = 1 if t else 0
            rows = sum(touch)
            o = out.contents
            o.rows, o.solved, o.points_solved = rows, rows, 2 * rows
            o.starts[0] = 0
            for k in range(1, 35):
                o.starts[k] = rows
            self.prev = list(zip(ab, touch))
            self.last = (n, rows)
            if self.calls == self.move_on:
                # send some awake bodies far away: their pairs' boxes stop meeting next step, they are
                # removed and the last pairs of the list move into their slots
                for i in range(min(self.moved, B.awake_count)):
                    s = B.awake_list[i]
                    B.position[3 * s] += 500.0
            self.calls += 1
            return 0
        except Exception as e:  # a ctypes callback cannot raise through C
            self.problems.append(repr(e))
            return -1


def world_with(stand_in, build):
    w = World({}, solver=oracle_io.solver(0))
    build(w)
    assert w._lib.bw_set_contact_step(w._w, C.cast(stand_in.fn, C.c_void_p), None) == 0
    return w


@pytest.mark.parametrize("build", [lambda w: scenes.pyramid(w, rows=10), lambda w: scenes.pile(w, count=400, seed=3, extent=8.0)],
                         ids=["pyramid", "pile400"])
def test_records_follow_their_pairs(build):
    s = StandIn()
    w = world_with(s, build)
    pairs_before = None
    for i in range(8):
        w.step(DT)
        if i == s.move_on:
            pairs_before = w.stats()["pairs"]
    assert not s.problems, s.problems[:5]
    assert s.calls == 8 and s.carried > 0
    st = w.stats()
    assert st["rows"] == s.last[1] and st["solved"] == s.last[1] and st["points"] == 2 * s.last[1]
    assert st["step"] == 8 and st["colours"] == (1 if s.last[1] else 0)
    assert st["pairs"] < pairs_before   # the moved bodies' pairs were removed
    w.destroy()


def test_set_after_stepping_and_begin_step_are_refused():
    s = StandIn()
    w = World({}, solver=oracle_io.solver(0))
    scenes.stack(w, count=3)
    w.step(DT)
    assert w._lib.bw_set_contact_step(w._w, C.cast(s.fn, C.c_void_p), None) == _ffi.BG_EINVAL
    w.destroy()
    w = world_with(s, lambda w: scenes.stack(w, count=3))
    with pytest.raises(BearingError):
        w.begin_step(DT)
    w.step(DT)
    assert s.calls == 1 and not s.problems
    w.destroy()


def test_a_failed_contact_step_fails_the_step():
    def failing(user, bodies, materials, pairs, step, out):
        return _ffi.BG_ECUDA
    bad = PROTO(failing)
    w = World({}, solver=oracle_io.solver(0))
    scenes.pyramid(w, rows=4)
    assert w._lib.bw_set_contact_step(w._w, C.cast(bad, C.c_void_p), None) == 0
    with pytest.raises(BearingError, match="contact step failed"):
        w.step(DT)
    assert w.stats()["step"] == 0   # no stats from the failed step
    w.destroy()


def test_no_pairs_still_steps():
    s = StandIn()
    w = world_with(s, lambda w: w.addBody({"position": (0.0, 5.0, 0.0)}))
    for _ in range(3):
        w.step(DT)
    assert s.calls == 3 and s.last == (0, 0) and not s.problems
    assert w.stats()["rows"] == 0 and w.stats()["colours"] == 0
    w.destroy()
