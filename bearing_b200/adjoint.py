"""Gradients through many worlds' steps: the backward pass of World.step for a batch of worlds.

The reference has no derivatives; this is the backward pass a differentiable World takes through
its steps.  A loss on the worlds' state after the last step is differentiated with respect to the
state before the first step and to every body's friction and restitution (World._friction,
_restitution, which emit() mixes per pair: src/contact.js:901-905).

Each step is the host side's narrowphase, emit, basis and carry (libbearing_host.so), the solve
stage on the GPU, and keep() into the pairs' memory.  The backward pass runs the steps again from
checkpoints and then in reverse, each step's reverse in three parts:

  bw_keep_backward     keep()'s reverse: the memory's adjoints onto the rows' results;
  bg_backward          the solve stage's reverse on the GPU (bearing_gpu.h), which recomputes the
                       step with records and sweeps its passes backwards;
  bw_narrow_backward   the narrowphase, emit, basis and carry's reverse: the rows' input adjoints
                       onto the bodies' poses, the materials and the memory carried in.

What the step decides (which pairs meet, the rows' order and colours, the points each block LCP
pushes, the clamps that hold) stays as the step took it: the gradient is that of the step's own
active set.  Checkpoints are taken every `checkpoint` steps (World copies, bw_clone); the steps
between two are run once more during the reverse, their inputs kept only for that segment.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import _ffi

BODY_GRAD = [("position", 3), ("rotation", 4), ("velocity", 3), ("angular", 3), ("tumbled", 3), ("ceiling", 1)]
ROW_GRAD = [("normal_impulse", 4), ("tangent_impulse1", 1), ("tangent_impulse2", 1), ("roll_impulse1", 1),
            ("roll_impulse2", 1), ("spin_impulse", 1), ("drift1", 1), ("drift2", 1), ("normal", 3), ("t1", 3),
            ("t2", 3), ("friction", 1), ("restitution", 1), ("separation", 4), ("point", 12)]
_PD = C.POINTER(C.c_double)


class Grads:
    """Adjoint arrays (numpy) for `count` slots or rows, with the ctypes structure over them."""

    def __init__(self, kind, count, arrays=None):
        fields = BODY_GRAD if kind == "body" else ROW_GRAD
        self.kind, self.count = kind, count
        self.a = arrays if arrays is not None else {f: np.zeros(k * max(count, 1)) for f, k in fields}
        self.s = (_ffi.BodyGrads if kind == "body" else _ffi.RowGrads)()
        for f, _ in fields:
            setattr(self.s, f, self.a[f].ctypes.data_as(_PD))

    def __getitem__(self, f):
        return self.a[f]


class _Record:
    """One step's solve-stage input for the whole batch (copies), with its rows' memory."""

    _BODY = [("position", np.float64, 3), ("rotation", np.float64, 4), ("velocity", np.float64, 3),
             ("angular", np.float64, 3), ("tumbled", np.float64, 3), ("ceiling", np.float64, 1),
             ("start", np.float64, 3), ("start_q", np.float64, 4), ("inv_i", np.float64, 6),
             ("inv_mass", np.float64, 1), ("inertia", np.float64, 3), ("inv_inertia", np.float64, 3),
             ("dims", np.float64, 3), ("damping", np.float64, 1), ("angular_damping", np.float64, 1),
             ("gravity_scale", np.float64, 1), ("type", np.uint8, 1), ("shape", np.uint8, 1),
             ("frozen", np.uint8, 1), ("framed", np.uint8, 1), ("lock", np.uint8, 1), ("joint_head", np.int32, 1),
             ("awake", np.uint8, 1)]
    _ROW = [("row", np.int32, 1), ("a", np.int32, 1), ("b", np.int32, 1), ("points", np.uint8, 1),
            ("normal", np.float64, 3), ("t1", np.float64, 3), ("t2", np.float64, 3), ("friction", np.float64, 1),
            ("restitution", np.float64, 1), ("tolerance", np.float64, 1), ("patch", np.float64, 1),
            ("separation", np.float64, 4), ("point", np.float64, 12), ("shift", np.float64, 12),
            ("normal_impulse", np.float64, 4), ("tangent_impulse1", np.float64, 1),
            ("tangent_impulse2", np.float64, 1), ("roll_impulse1", np.float64, 1), ("roll_impulse2", np.float64, 1),
            ("spin_impulse", np.float64, 1), ("drift1", np.float64, 1), ("drift2", np.float64, 1),
            ("gap", np.float64, 1), ("max_normal_impulse", np.float64, 4), ("relative_velocity", np.float64, 4),
            ("sliding", np.uint8, 1), ("anchor_a", np.float64, 3), ("anchor_b", np.float64, 3)]
    _CT = {np.float64: C.c_double, np.uint8: C.c_uint8, np.int32: C.c_int32}

    def __init__(self, B, R, W, S, mem):
        def read(ptr, n, dt):
            return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True) if n else np.zeros(1, dt)
        self.nb, self.nr, self.nw = B.capacity, R.count, W.count
        self.na = B.awake_count
        self.awake_list = read(B.awake_list, self.na, np.int32)
        self.body = {f: read(getattr(B, f), k * self.nb, dt) for f, dt, k in self._BODY}
        self.rows = {f: read(getattr(R, f), k * self.nr, dt) for f, dt, k in self._ROW}
        self.offsets = {f: read(getattr(W, f), self.nw + 1, np.int32) for f in ("body_offset", "awake_offset",
                                                                                 "row_offset")}
        self.starts = read(W.starts, _ffi.BG_STARTS * self.nw, np.int32)
        self.dt, self.substeps, self.gravity = S.dt, S.substeps, tuple(S.gravity)
        self.mem = mem
        self.out = None

    # What keep() reads of the step's results.
    KEPT = ("normal_impulse", "tangent_impulse1", "tangent_impulse2", "roll_impulse1", "roll_impulse2",
            "spin_impulse", "drift1", "drift2")

    def keep_results(self, R):
        """After the solve stage: the results keep() reads."""
        k = dict((f, per) for f, _, per in self._ROW)
        self.out = {f: np.ctypeslib.as_array(getattr(R, f), shape=(k[f] * self.nr,)).copy() if self.nr else
                    np.zeros(1) for f in self.KEPT}

    # What the solve stage's reverse writes (the recomputed step's results), per bg_bodies / bg_rows.
    WRITTEN_BODY = ("position", "rotation", "velocity", "angular", "tumbled", "ceiling", "start", "start_q", "inv_i")
    WRITTEN_ROW = KEPT + ("gap", "max_normal_impulse", "relative_velocity", "sliding", "anchor_a", "anchor_b")

    def views(self, results=False, writable=False):
        """bg_bodies / bg_rows / bg_worlds / bg_step over the record's arrays: with `writable`, over
        copies of the columns the solve stage's reverse writes its recomputed results into (the
        rest are only read, and shared); with `results`, the rows carry the step's results where
        keep() reads them."""
        body = {f: v.copy() if writable and f in self.WRITTEN_BODY else v for f, v in self.body.items()}
        rows = {f: v.copy() if writable and f in self.WRITTEN_ROW else v for f, v in self.rows.items()}
        if results:
            rows.update(self.out)
        keep = [body, rows]
        B, R, W = _ffi.Bodies(), _ffi.Rows(), _ffi.Worlds()
        B.capacity, B.awake_count = self.nb, self.na
        B.awake_list = self.awake_list.ctypes.data_as(C.POINTER(C.c_int32))
        for f, dt, _ in self._BODY:
            setattr(B, f, body[f].ctypes.data_as(C.POINTER(self._CT[dt])))
        R.count = self.nr
        R.solved = 0
        for f, dt, _ in self._ROW:
            setattr(R, f, rows[f].ctypes.data_as(C.POINTER(self._CT[dt])))
        W.count = self.nw
        for f in ("body_offset", "awake_offset", "row_offset"):
            setattr(W, f, self.offsets[f].ctypes.data_as(C.POINTER(C.c_int32)))
        W.starts = self.starts.ctypes.data_as(C.POINTER(C.c_int32))
        W.gravity = None
        S = _ffi.Step(self.dt, self.substeps, (C.c_double * 3)(*self.gravity))
        return B, R, W, S, keep

    def keys(self):
        """Each row's pair as one integer: world, then the two slots (world-local)."""
        world = np.repeat(np.arange(self.nw, dtype=np.int64), np.diff(self.offsets["row_offset"]))
        a = self.rows["a"][: self.nr].astype(np.int64)
        b = self.rows["b"][: self.nr].astype(np.int64)
        return (world << 40) | (a << 20) | b


class _Memory:
    """bw_row_memory arrays for `n` rows."""

    def __init__(self, n):
        n1 = max(n, 1)
        self.pid = np.zeros(4 * n1, np.uint32)
        self.margin = np.zeros(n1)
        self.remembered = np.zeros(n1, np.uint8)
        self.memory_pid = np.zeros(4 * n1, np.uint32)
        self.memory = np.zeros(_ffi.BW_MEMORY * n1)
        self.s = _ffi.RowMemory(self.pid.ctypes.data_as(C.POINTER(C.c_uint32)), self.margin.ctypes.data_as(_PD),
                                self.remembered.ctypes.data_as(C.POINTER(C.c_uint8)),
                                self.memory_pid.ctypes.data_as(C.POINTER(C.c_uint32)),
                                self.memory.ctypes.data_as(_PD))


def _host_threads():
    """The host threads this process may run on (its CPU affinity, which may be fewer than the
    machine's CPUs)."""
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return os.cpu_count() or 1


class BatchBackward:
    """Steps a list of Worlds together (their host sides on the CPU, their solve stages as one batch
    on the GPU) and differentiates a loss on their final state.  The worlds are left in their
    final state."""

    def __init__(self, worlds, dt, device=0, threads=None):
        self.worlds = list(worlds)
        self.dt = float(dt)
        self.host = _ffi.host()
        self.gpu = _ffi.gpu()
        self.ctx = self.gpu.bg_create(device, 0)
        if not self.ctx:
            raise RuntimeError(f"bg_create({device}) failed: no usable CUDA device")
        self.threads = threads or _host_threads()
        handles = (C.c_void_p * len(self.worlds))(*[w._w for w in self.worlds])
        self.batch = self.host.bw_batch_create(handles, len(self.worlds))
        counts = [w._count for w in self.worlds]
        self.body_offset = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        self.nb = int(self.body_offset[-1])
        self.friction = np.zeros(max(self.nb, 1))
        self.restitution = np.zeros(max(self.nb, 1))
        for w, o in zip(self.worlds, self.body_offset[:-1]):
            fr, re = np.zeros(w._count), np.zeros(w._count)
            self.host.bw_materials(w._w, fr.ctypes.data_as(_PD), re.ctypes.data_as(_PD))
            self.friction[o: o + w._count] = fr
            self.restitution[o: o + w._count] = re
        self.gravity = np.zeros(3)
        self.device_ms = 0.0
        self.device_bytes = 0
        self.tape_peak = 0
        # host seconds of the backward pass, by part (bg_backward's is its wall time, kernel included)
        self.times = {"recompute": 0.0, "keep_backward": 0.0, "stage_backward": 0.0, "narrow_backward": 0.0}

    def close(self):
        if self.batch:
            self.host.bw_batch_destroy(self.batch)
            self.batch = None
        if self.ctx:
            self.gpu.bg_destroy(self.ctx)
            self.ctx = None

    def _step(self, record=False):
        h, g = self.host, self.gpu
        if h.bw_batch_begin_step(self.batch, self.dt, self.threads) != 0:
            raise RuntimeError("bw_batch_begin_step failed")
        B, R, W, S = _ffi.Bodies(), _ffi.Rows(), _ffi.Worlds(), _ffi.Step()
        h.bw_batch_views(self.batch, C.byref(B), C.byref(R), C.byref(W), C.byref(S))
        self.gravity[:] = S.gravity
        rec = None
        if record:
            mem = _Memory(R.count)
            if h.bw_batch_row_memory(self.batch, C.byref(mem.s)) != 0:
                raise RuntimeError("bw_batch_row_memory failed")
            rec = _Record(B, R, W, S, mem)
        rc = g.bg_batch_solve_step(self.ctx, C.byref(B), C.byref(R), C.byref(W), C.byref(S))
        if rc != 0:
            raise RuntimeError(f"bg_batch_solve_step: {rc} {g.bg_last_error(self.ctx).decode()}")
        if rec is not None:
            rec.keep_results(R)
        if h.bw_batch_end_step(self.batch, self.threads) != 0:
            raise RuntimeError("bw_batch_end_step failed")
        return rec

    def forward(self, steps, checkpoint=20):
        """`steps` steps, copying every world every `checkpoint` steps (for backward)."""
        self.steps, self.checkpoint = steps, checkpoint
        self.checkpoints = {}
        for k in range(steps):
            if k % checkpoint == 0:
                self.checkpoints[k] = [self.host.bw_clone(w._w) for w in self.worlds]
            self._step()

    def _reverse_step(self, rec, bar, mem_next, grad_fr, grad_re):
        t0 = time.perf_counter()
        nr = rec.nr
        mem_after = np.zeros(_ffi.BW_MEMORY * max(nr, 1))
        keys = rec.keys()
        if mem_next is not None and nr:
            next_keys, next_bar = mem_next
            if next_keys.size:
                order = np.argsort(next_keys, kind="stable")
                sk = next_keys[order]
                at = np.clip(np.searchsorted(sk, keys), 0, sk.size - 1)
                hit = sk[at] == keys
                mb = next_bar.reshape(-1, _ffi.BW_MEMORY)
                ma = mem_after.reshape(-1, _ffi.BW_MEMORY)
                ma[np.flatnonzero(hit)] = mb[order[at[hit]]]
        B, R, W, S, keep = rec.views(results=True)
        seed = Grads("row", nr)
        if self.host.bw_keep_backward(C.byref(R), C.byref(W), mem_after.ctypes.data_as(_PD), C.byref(seed.s)) != 0:
            raise RuntimeError("bw_keep_backward failed")
        t1 = time.perf_counter()
        B, R, W, S, keep = rec.views(writable=True)
        body_grad, row_grad = Grads("body", self.nb), Grads("row", nr)
        rc = self.gpu.bg_backward(self.ctx, C.byref(B), C.byref(R), C.byref(W), C.byref(S), C.byref(bar.s),
                                  C.byref(seed.s), C.byref(body_grad.s), C.byref(row_grad.s))
        if rc != 0:
            raise RuntimeError(f"bg_backward: {rc} {self.gpu.bg_last_error(self.ctx).decode()}")
        self.device_ms += self.gpu.bg_backward_ms(self.ctx)
        self.device_bytes += self.gpu.bg_backward_bytes(self.ctx)
        self.tape_peak = max(self.tape_peak, self.gpu.bg_backward_tape_peak(self.ctx))
        for f in ("normal", "t1", "t2"):   # keep() read these too
            row_grad[f][: 3 * nr] += seed[f][: 3 * nr]
        t2 = time.perf_counter()
        B, R, W, S, keep = rec.views()   # the step's input, untouched
        mem_before = np.zeros(_ffi.BW_MEMORY * max(nr, 1))
        rc = self.host.bw_narrow_backward(C.byref(B), C.byref(R), C.byref(W), C.byref(rec.mem.s),
                                          self.gravity.ctypes.data_as(_PD), self.friction.ctypes.data_as(_PD),
                                          self.restitution.ctypes.data_as(_PD), C.byref(row_grad.s),
                                          body_grad["position"].ctypes.data_as(_PD),
                                          body_grad["rotation"].ctypes.data_as(_PD), grad_fr.ctypes.data_as(_PD),
                                          grad_re.ctypes.data_as(_PD), mem_before.ctypes.data_as(_PD), self.threads)
        if rc != 0:
            raise RuntimeError(f"bw_narrow_backward: {rc}")
        t3 = time.perf_counter()
        self.times["keep_backward"] += t1 - t0
        self.times["stage_backward"] += t2 - t1
        self.times["narrow_backward"] += t3 - t2
        return body_grad, (keys, mem_before[: _ffi.BW_MEMORY * nr])

    def backward(self, seed):
        """`seed`: the loss's adjoints of the final body state, a dict of BODY_GRAD columns over the
        batch's slots (missing columns are 0).  Returns (adjoints of the initial body state,
        adjoints of each slot's friction, of each slot's restitution)."""
        bar = Grads("body", self.nb)
        for f, _ in BODY_GRAD:
            if f in seed:
                bar[f][: seed[f].size] = seed[f]
        grad_fr = np.zeros(max(self.nb, 1))
        grad_re = np.zeros(max(self.nb, 1))
        final = [self.host.bw_clone(w._w) for w in self.worlds]
        mem_next = None
        try:
            for c0 in sorted(self.checkpoints, reverse=True):
                for w, snap in zip(self.worlds, self.checkpoints[c0]):
                    self.host.bw_copy(w._w, snap)
                t0 = time.perf_counter()
                recs = [self._step(record=True) for _ in range(c0, min(c0 + self.checkpoint, self.steps))]
                self.times["recompute"] += time.perf_counter() - t0
                for rec in reversed(recs):
                    bar, mem_next = self._reverse_step(rec, bar, mem_next, grad_fr, grad_re)
        finally:
            for w, snap in zip(self.worlds, final):
                self.host.bw_copy(w._w, snap)
                self.host.bw_destroy(snap)
            for snaps in self.checkpoints.values():
                for snap in snaps:
                    self.host.bw_destroy(snap)
            self.checkpoints = {}
        return bar, grad_fr[: self.nb], grad_re[: self.nb]


def tower_gradients(count, seed=5000, steps=120, dt=1 / 60, checkpoint=20, first=0, device=0):
    """The differentiable workload: `count` towers struck by a ball (scenes.tower, world i drawn
    from scenes.batch_rng(seed, first + i)), stepped `steps` times as one batch, and the gradient
    of each tower's loss (scenes.tower_loss) with respect to its friction, its restitution and the
    ball's launch velocity (3).  Returns a dict: gradients (count x 5), losses, the final positions,
    and timings (forward and backward seconds, the adjoint kernels' device milliseconds)."""
    from . import scenes
    from .world import World

    worlds, infos = [], []
    for i in range(count):
        w = World({}, solver=(0, 0))   # no solver of its own: stepped only as part of the batch
        _, info = scenes.tower(w, scenes.batch_rng(seed, first + i))
        worlds.append(w)
        infos.append(info)
    bb = BatchBackward(worlds, dt, device=device)
    try:
        t0 = time.perf_counter()
        bb.forward(steps, checkpoint)
        t1 = time.perf_counter()
        position = np.concatenate([w.state()["position"] for w in worlds])
        losses, seed_p = [], np.zeros_like(position)
        for w, info, o in zip(worlds, infos, bb.body_offset[:-1]):
            loss, s = scenes.tower_loss(position, info, int(o))
            losses.append(loss)
            seed_p += s
        bar, g_fr, g_re = bb.backward({"position": seed_p})
        t2 = time.perf_counter()
        grads = np.zeros((count, 5))
        for i, (w, info, o) in enumerate(zip(worlds, infos, bb.body_offset[:-1])):
            o = int(o)
            grads[i, 0] = g_fr[o: o + w._count].sum()
            grads[i, 1] = g_re[o: o + w._count].sum()
            ball = o + info["ball"]
            grads[i, 2:] = bar["velocity"][3 * ball: 3 * ball + 3]
        return dict(gradients=grads, losses=np.array(losses), position=position, forward_s=t1 - t0,
                    backward_s=t2 - t1, device_ms=bb.device_ms, device_bytes=bb.device_bytes, tape_peak=bb.tape_peak,
                    infos=infos,
                    backward_parts=dict(bb.times))
    finally:
        bb.close()
        for w in worlds:
            w.destroy()

