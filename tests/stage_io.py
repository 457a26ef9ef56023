"""Copies of a solve stage's input, for running the same step through two solvers.

``StageCopy(world)`` takes the solve stage's input as the world's host side left it (after
``world.begin_step``) into numpy arrays of its own; ``views()`` gives bg_bodies / bg_rows /
bg_step structures over those arrays, which the CUDA library and the oracle both accept.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from bearing_b200 import _ffi

# (field, numpy dtype, numbers per slot)
BODY_COLUMNS = [
    ("position", np.float64, 3), ("rotation", np.float64, 4), ("velocity", np.float64, 3),
    ("angular", np.float64, 3), ("tumbled", np.float64, 3), ("ceiling", np.float64, 1),
    ("start", np.float64, 3), ("start_q", np.float64, 4), ("inv_i", np.float64, 6),
    ("inv_mass", np.float64, 1), ("inertia", np.float64, 3), ("inv_inertia", np.float64, 3),
    ("dims", np.float64, 3), ("damping", np.float64, 1), ("angular_damping", np.float64, 1),
    ("gravity_scale", np.float64, 1), ("type", np.uint8, 1), ("shape", np.uint8, 1),
    ("frozen", np.uint8, 1), ("framed", np.uint8, 1), ("lock", np.uint8, 1), ("joint_head", np.int32, 1),
    ("awake", np.uint8, 1),
]
# (field, numpy dtype, numbers per row)
ROW_COLUMNS = [
    ("row", np.int32, 1), ("a", np.int32, 1), ("b", np.int32, 1), ("points", np.uint8, 1),
    ("normal", np.float64, 3), ("t1", np.float64, 3), ("t2", np.float64, 3), ("friction", np.float64, 1),
    ("restitution", np.float64, 1), ("tolerance", np.float64, 1), ("patch", np.float64, 1),
    ("separation", np.float64, 4), ("point", np.float64, 12), ("shift", np.float64, 12),
    ("normal_impulse", np.float64, 4), ("tangent_impulse1", np.float64, 1), ("tangent_impulse2", np.float64, 1),
    ("roll_impulse1", np.float64, 1), ("roll_impulse2", np.float64, 1), ("spin_impulse", np.float64, 1),
    ("drift1", np.float64, 1), ("drift2", np.float64, 1), ("gap", np.float64, 1),
    ("max_normal_impulse", np.float64, 4), ("relative_velocity", np.float64, 4), ("sliding", np.uint8, 1),
    ("anchor_a", np.float64, 3), ("anchor_b", np.float64, 3),
]
# What the solve stage writes.
BODY_OUT = ["position", "rotation", "velocity", "angular", "tumbled", "ceiling", "start", "start_q", "inv_i"]
ROW_OUT = ["normal_impulse", "tangent_impulse1", "tangent_impulse2", "roll_impulse1", "roll_impulse2",
           "spin_impulse", "drift1", "drift2", "gap", "max_normal_impulse", "relative_velocity"]
# Written for solved rows only.
ROW_OUT_SOLVED = ["sliding", "anchor_a", "anchor_b"]

_CT = {np.float64: C.c_double, np.uint8: C.c_uint8, np.int32: C.c_int32}


def _ptr(arr, dtype):
    return arr.ctypes.data_as(C.POINTER(_CT[dtype]))


def _read(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


class StageCopy:
    """A solve stage's input, in arrays of its own."""

    def __init__(self, world=None, *, arrays=None, views=None):
        if arrays is not None:
            self.__dict__.update(arrays)
            return
        B, R, S = views if views is not None else world.views()
        self.capacity = B.capacity
        self.awake_count = B.awake_count
        self.awake_list = _read(B.awake_list, B.awake_count, np.int32)
        self.body = {f: _read(getattr(B, f), per * B.capacity, dt) for f, dt, per in BODY_COLUMNS}
        self.count = R.count
        self.solved = R.solved
        self.starts = np.array(list(R.starts), dtype=np.int32)
        self.rows = {f: _read(getattr(R, f), per * R.count, dt) for f, dt, per in ROW_COLUMNS}
        self.dt = S.dt
        self.substeps = S.substeps
        self.gravity = tuple(S.gravity)

    def copy(self):
        return StageCopy(arrays=dict(
            capacity=self.capacity, awake_count=self.awake_count, awake_list=self.awake_list.copy(),
            body={k: v.copy() for k, v in self.body.items()}, count=self.count, solved=self.solved,
            starts=self.starts.copy(), rows={k: v.copy() for k, v in self.rows.items()}, dt=self.dt,
            substeps=self.substeps, gravity=self.gravity))

    def save(self, path):
        """Every array and count into one .npz file (StageCopy.load reads it back)."""
        arrays = {"b_" + k: v for k, v in self.body.items()}
        arrays.update({"r_" + k: v for k, v in self.rows.items()})
        np.savez(path, awake_list=self.awake_list, starts=self.starts, gravity=np.asarray(self.gravity),
                 counts=np.array([self.capacity, self.awake_count, self.count, self.solved, self.substeps]),
                 dt=np.array([self.dt]), **arrays)

    @staticmethod
    def load(path):
        z = np.load(path)
        capacity, awake_count, count, solved, substeps = (int(x) for x in z["counts"])
        return StageCopy(arrays=dict(
            capacity=capacity, awake_count=awake_count, awake_list=z["awake_list"].copy(),
            body={k[2:]: z[k].copy() for k in z.files if k.startswith("b_")}, count=count, solved=solved,
            starts=z["starts"].copy(), rows={k[2:]: z[k].copy() for k in z.files if k.startswith("r_")},
            dt=float(z["dt"][0]), substeps=substeps, gravity=tuple(float(x) for x in z["gravity"])))

    def pinned(self):
        """The same arrays in page-locked host memory (torch's pinned allocator), which the CUDA
        library copies to and from directly."""
        import torch

        keep = []

        def pin(arr):
            t = torch.empty(max(arr.size, 1), dtype=getattr(torch, arr.dtype.name)).pin_memory()
            keep.append(t)
            out = t.numpy()[: arr.size]
            out[:] = arr
            return out

        c = StageCopy(arrays=dict(
            capacity=self.capacity, awake_count=self.awake_count, awake_list=pin(self.awake_list),
            body={k: pin(v) for k, v in self.body.items()}, count=self.count, solved=self.solved,
            starts=self.starts.copy(), rows={k: pin(v) for k, v in self.rows.items()}, dt=self.dt,
            substeps=self.substeps, gravity=self.gravity))
        c._pinned = keep
        return c

    def fill(self, other):
        """Copies other's values into these arrays (same sizes)."""
        np.copyto(self.awake_list, other.awake_list)
        for k, v in other.body.items():
            np.copyto(self.body[k], v)
        for k, v in other.rows.items():
            np.copyto(self.rows[k], v)

    def views(self):
        B = _ffi.Bodies()
        B.capacity = self.capacity
        B.awake_count = self.awake_count
        B.awake_list = _ptr(self.awake_list, np.int32)
        for f, dt, _ in BODY_COLUMNS:
            setattr(B, f, _ptr(self.body[f], dt))
        R = _ffi.Rows()
        R.count = self.count
        R.solved = self.solved
        R.starts = (C.c_int32 * _ffi.BG_STARTS)(*[int(x) for x in self.starts])
        for f, dt, _ in ROW_COLUMNS:
            setattr(R, f, _ptr(self.rows[f], dt))
        S = _ffi.Step(self.dt, self.substeps, (C.c_double * 3)(*self.gravity))
        self._keep = (B, R, S)
        return B, R, S


def _first_unequal(x, y):
    """Index of the first entry where x and y differ, or None.  Floats compare bit for bit, except
    that a NaN matches any NaN: the CPU's and the GPU's default NaN payloads differ, and a NaN's
    payload is not a result."""
    if x.dtype == np.float64:
        nx, ny = np.isnan(x), np.isnan(y)
        unequal = (x.view(np.uint64) != y.view(np.uint64)) & ~(nx & ny)
    else:
        unequal = x != y
    hit = np.flatnonzero(unequal)
    return int(hit[0]) if hit.size else None


def first_difference(a: StageCopy, b: StageCopy):
    """None if every column the solve stage writes is bit-identical (NaN matching NaN); else a
    description of the first difference."""
    for f in BODY_OUT:
        i = _first_unequal(a.body[f], b.body[f])
        if i is not None:
            return f"body {f}[{i}]: {a.body[f][i]!r} vs {b.body[f][i]!r}"
    per = dict((f, p) for f, _, p in ROW_COLUMNS)
    for f in ROW_OUT:
        i = _first_unequal(a.rows[f], b.rows[f])
        if i is not None:
            return f"row {f}[{i}] (row {i // per[f]}): {a.rows[f][i]!r} vs {b.rows[f][i]!r}"
    n = a.solved
    for f in ROW_OUT_SOLVED:
        k = per[f]
        x, y = a.rows[f][: k * n], b.rows[f][: k * n]
        i = _first_unequal(x, y)
        if i is not None:
            return f"row {f}[{i}] (row {i // k}): {x[i]!r} vs {y[i]!r}"
    return None


def max_relative_difference(a: StageCopy, b: StageCopy) -> float:
    worst = 0.0
    for f in BODY_OUT:
        x, y = a.body[f], b.body[f]
        d = np.abs(x - y) / np.maximum(1.0, np.maximum(np.abs(x), np.abs(y)))
        if d.size:
            worst = max(worst, float(np.nanmax(d)))
    return worst


class BatchCopy:
    """A batch's solve-stage input (bw_batch_views: every world's arrays end to end, and the table
    of where each world's part starts) in arrays of its own."""

    def __init__(self, B, R, W, S):
        self.stage = StageCopy(views=(B, R, S))
        n = W.count
        self.worlds = n
        self.body_offset = _read(W.body_offset, n + 1, np.int32)
        self.awake_offset = _read(W.awake_offset, n + 1, np.int32)
        self.row_offset = _read(W.row_offset, n + 1, np.int32)
        self.starts = _read(W.starts, _ffi.BG_STARTS * n, np.int32)

    def copy(self):
        c = BatchCopy.__new__(BatchCopy)
        c.stage = self.stage.copy()
        c.worlds = self.worlds
        for k in ("body_offset", "awake_offset", "row_offset", "starts"):
            setattr(c, k, getattr(self, k).copy())
        return c

    def fill(self, other):
        self.stage.fill(other.stage)

    def pinned(self):
        """The same batch with its columns in page-locked host memory (see StageCopy.pinned)."""
        c = BatchCopy.__new__(BatchCopy)
        c.stage = self.stage.pinned()
        c.worlds = self.worlds
        for k in ("body_offset", "awake_offset", "row_offset", "starts"):
            setattr(c, k, getattr(self, k).copy())
        return c

    def views(self):
        B, R, S = self.stage.views()
        W = _ffi.Worlds(self.worlds, _ptr(self.body_offset, np.int32), _ptr(self.awake_offset, np.int32),
                        _ptr(self.row_offset, np.int32), _ptr(self.starts, np.int32), None)
        self._keep = (B, R, W, S)
        return B, R, W, S

    def world(self, i):
        """World i's part as a StageCopy of its own (the batch keeps slots and rows world-local)."""
        b0, b1 = int(self.body_offset[i]), int(self.body_offset[i + 1])
        a0, a1 = int(self.awake_offset[i]), int(self.awake_offset[i + 1])
        r0, r1 = int(self.row_offset[i]), int(self.row_offset[i + 1])
        st = self.stage
        starts = self.starts[_ffi.BG_STARTS * i: _ffi.BG_STARTS * (i + 1)].copy()
        return StageCopy(arrays=dict(
            capacity=b1 - b0, awake_count=a1 - a0, awake_list=st.awake_list[a0:a1].copy(),
            body={f: st.body[f][per * b0: per * b1].copy() for f, _, per in BODY_COLUMNS},
            count=r1 - r0, solved=int(starts[33]), starts=starts,
            rows={f: st.rows[f][per * r0: per * r1].copy() for f, _, per in ROW_COLUMNS},
            dt=st.dt, substeps=st.substeps, gravity=st.gravity))

    def save(self, path):
        """The batch's arrays and its table of worlds into one .npz file (BatchCopy.load reads it)."""
        base = str(path)
        self.stage.save(base + ".stage.npz")
        np.savez(base, body_offset=self.body_offset, awake_offset=self.awake_offset, row_offset=self.row_offset,
                 starts=self.starts)

    @staticmethod
    def load(path):
        base = str(path)
        z = np.load(base if base.endswith(".npz") else base + ".npz")
        c = BatchCopy.__new__(BatchCopy)
        c.stage = StageCopy.load(base + ".stage.npz")
        for k in ("body_offset", "awake_offset", "row_offset", "starts"):
            setattr(c, k, z[k].copy())
        c.worlds = len(c.body_offset) - 1
        return c

    def subset(self, indices):
        """A batch of only the worlds `indices`, in that order (their parts laid end to end)."""
        parts = [self.world(int(i)) for i in indices]
        c = BatchCopy.__new__(BatchCopy)
        c.worlds = len(parts)
        st = self.stage
        c.body_offset = np.cumsum([0] + [p.capacity for p in parts]).astype(np.int32)
        c.awake_offset = np.cumsum([0] + [p.awake_count for p in parts]).astype(np.int32)
        c.row_offset = np.cumsum([0] + [p.count for p in parts]).astype(np.int32)
        c.starts = np.concatenate([p.starts for p in parts]).astype(np.int32)
        c.stage = StageCopy(arrays=dict(
            capacity=int(c.body_offset[-1]), awake_count=int(c.awake_offset[-1]),
            awake_list=np.concatenate([p.awake_list for p in parts]).astype(np.int32),
            body={f: np.concatenate([p.body[f] for p in parts]) for f, _, _ in BODY_COLUMNS},
            count=int(c.row_offset[-1]), solved=0, starts=np.zeros(_ffi.BG_STARTS, np.int32),
            rows={f: np.concatenate([p.rows[f] for p in parts]) for f, _, _ in ROW_COLUMNS},
            dt=st.dt, substeps=st.substeps, gravity=st.gravity))
        return c

    def part(self, i, out):
        """Writes StageCopy `out` (world i's part, solved alone) back over this batch's arrays."""
        b0, b1 = int(self.body_offset[i]), int(self.body_offset[i + 1])
        r0, r1 = int(self.row_offset[i]), int(self.row_offset[i + 1])
        for f, _, per in BODY_COLUMNS:
            self.stage.body[f][per * b0: per * b1] = out.body[f]
        for f, _, per in ROW_COLUMNS:
            self.stage.rows[f][per * r0: per * r1] = out.rows[f]
