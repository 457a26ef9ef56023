"""Pair lists and manifolds for the narrowphase entry points (bw_narrow_pairs, bw_collide_pairs,
bg_collide): numpy arrays of their own behind bg_pairs / bg_manifolds structures."""
from __future__ import annotations

import ctypes as C

import numpy as np

from bearing_b200 import _ffi

P = _ffi.BG_POINTS
_PD = C.POINTER(C.c_double)


class PairList:
    """A copy of a bg_pairs list."""

    def __init__(self, view: _ffi.Pairs):
        n = view.count
        self.count = n

        def read(ptr, dt):
            return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True) if n else np.zeros(1, dt)

        self.a, self.b = read(view.a, np.int32), read(view.b, np.int32)
        self.margin, self.tolerance = read(view.margin, np.float64), read(view.tolerance, np.float64)

    def view(self) -> _ffi.Pairs:
        self._s = _ffi.Pairs(self.count, self.a.ctypes.data_as(C.POINTER(C.c_int32)),
                             self.b.ctypes.data_as(C.POINTER(C.c_int32)), self.margin.ctypes.data_as(_PD),
                             self.tolerance.ctypes.data_as(_PD))
        return self._s


class ManifoldSet:
    """bg_manifolds over arrays for n pairs."""

    def __init__(self, n: int, fill=0):
        n1 = max(n, 1)
        self.n = n
        self.points = np.full(n1, fill, np.uint8)
        self.normal = np.full(3 * n1, fill, np.float64)
        self.point = np.full(3 * P * n1, fill, np.float64)
        self.separation = np.full(P * n1, fill, np.float64)
        self.pid = np.full(P * n1, fill, np.uint32)
        self.s = _ffi.Manifolds(self.points.ctypes.data_as(C.POINTER(C.c_uint8)), self.normal.ctypes.data_as(_PD),
                                self.point.ctypes.data_as(_PD), self.separation.ctypes.data_as(_PD),
                                self.pid.ctypes.data_as(C.POINTER(C.c_uint32)))

    def columns(self):
        return {"points": self.points[: self.n], "normal": self.normal[: 3 * self.n],
                "point": self.point[: 3 * P * self.n], "separation": self.separation[: P * self.n],
                "pid": self.pid[: P * self.n]}


def first_unequal(x: ManifoldSet, y: ManifoldSet):
    """The first column and pair where two manifold sets differ in their bytes, or None."""
    cx, cy = x.columns(), y.columns()
    for f in cx:
        if cx[f].tobytes() != cy[f].tobytes():
            per = cx[f].size // max(x.n, 1)
            diff = np.flatnonzero(cx[f].view(f"u{cx[f].itemsize}") != cy[f].view(f"u{cy[f].itemsize}"))
            i = int(diff[0])
            return f"{f} of pair {i // per}: {cx[f][i]!r} vs {cy[f][i]!r}"
    return None


def world_pairs(world) -> PairList:
    """The pairs the world's last bw_begin_step handed to collide()."""
    view = _ffi.Pairs()
    assert _ffi.host().bw_narrow_pairs(world._w, C.byref(view)) == 0
    return PairList(view)


def host_collide(bodies, gravity, pairs: PairList, threads=4) -> ManifoldSet:
    out = ManifoldSet(pairs.count, fill=0xAB)
    g = np.asarray(gravity, np.float64)
    rc = _ffi.host().bw_collide_pairs(C.byref(bodies), g.ctypes.data_as(_PD), C.byref(pairs.view()), C.byref(out.s),
                                      threads)
    assert rc == 0, rc
    return out
