"""Benchmark: the contact solve stage of a 50,000-body mixed pile at step 300, on one B200.

A "step" here is one solve stage (src/world.js:962-1032: inertias, prepare, 8 substeps of
accelerate / warm / solve / move / relax, restitution, slipped) over the pile's manifolds at
step 301, the pile having been stepped 300 times first (host side of the step on the CPU, solve
stage on the GPU).  Metric: contact rows/s = solved rows x substeps x 3 (warm, solve and relax
row visits) / solve-stage seconds.

  value     the solve stage with its input resident in HBM: bg_restore (untimed), an L2 flush
            (untimed), then CUDA events around bg_solve on the library's stream
  e2e       the same solve stage through bg_solve_step with host arrays in page-locked memory:
            upload, solve and download inside the timed region, events on the same stream
  roofline  algorithmic bytes of one solve-stage kernel (counted from the rows' point counts by
            the rule in algorithmic_bytes()) / that kernel's event-timed duration, against the
            measured HBM copy bandwidth
  cpu_baseline  the CPU restatement of the reference's solve stage on this box's host cores
            (rank 0, N=1), on a bounded sample of the same input

--impl reference times that CPU solve stage alone, with every host thread, as the reference arm.
Under torchrun each rank solves its own replica of the pile (the solve stage of one world does
not shard: replicas only); value is the sum over ranks, time the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DT = 1 / 60
SUBSTEPS = 8


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--bodies", type=int, default=50_000)
    p.add_argument("--at", type=int, default=300, help="steps taken before the timed solve stage")
    p.add_argument("--cpu-sample", type=int, default=2, help="solve stages the CPU baseline times")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--resident-only", action="store_true", help="time the resident solve only (for profiling)")
    p.add_argument("--batch-worlds", type=int, default=4096, help="worlds in the batched-worlds measurement")
    p.add_argument("--batch-at", type=int, default=300, help="steps the batch takes before its timed solve stage")
    p.add_argument("--no-batch", action="store_true", help="skip the batched-worlds measurement")
    p.add_argument("--adjoint-worlds", type=int, default=1024, help="towers in the backward-pass measurement")
    p.add_argument("--adjoint-steps", type=int, default=120)
    p.add_argument("--no-adjoint", action="store_true", help="skip the backward-pass measurement")
    p.add_argument("--no-contact", action="store_true", help="skip the device contact-step measurement")
    p.add_argument("--save-batch", default=None, help="write the batch's timed input (files PATH.npz, PATH.stage.npz)")
    p.add_argument("--load-batch", default=None,
                   help="solve a batch written by --save-batch once on the persistent grid and exit (a profiler "
                        "then sees one launch of the batched kernel)")
    p.add_argument("--save-input", default=None, help="write the timed solve stage's input to this .npz")
    p.add_argument("--load-input", default=None,
                   help="time the solve stage of an input written by --save-input instead of building the pile "
                        "(a profiler then sees no launches of the pile's first steps)")
    return p.parse_args()


# ---- the workload -------------------------------------------------------------------------

def build_pile(solver, bodies, at, log=None):
    """The pile stepped `at` times with `solver`, then the host side of step at+1."""
    from bearing_b200 import scenes
    from bearing_b200.world import GpuSolver, World
    w = World({}, solver=solver)
    if isinstance(solver, GpuSolver):
        w.set_narrowphase(solver)   # the same rows as the host's narrowphase, found on the device
    scenes.pile(w, count=bodies, seed=50_000)
    t0 = time.time()
    for i in range(at):
        w.step(DT)
        if log and (i + 1) % 50 == 0:
            log(f"step {i + 1}: {w.stats()} ({time.time() - t0:.0f} s)")
    w.begin_step(DT)
    return w


def algorithmic_bytes(copy):
    """Bytes one solve stage must move at least: each column a pass needs read once and each
    column it writes written once, per row per pass, at the widths the rows are kept in, plus the
    two bodies' records each row reads and writes, plus the per-body passes.  FP64 = 8 bytes.

      warm    per row 521 + 56 n        (n = the row's points)
      solve   per row 754 + 160 n + 8 n^2, and 160 + 48 n more where the separation is not
              known (first substep) and in relax, which writes it (8 n)
      prepare per row 560 + 256 n + 8 n^2
      bodies  per awake body: 200 once, then 124 (accelerate) + 300 (move) a substep
      slipped per row 289 + 32 n
    """
    import numpy as np
    pts = copy.rows["points"][: copy.solved].astype(np.int64)
    n1 = int(pts.sum())
    n2 = int((pts * pts).sum())
    rows = copy.solved
    warm = 521 * rows + 56 * n1
    solve_known = 754 * rows + 160 * n1 + 8 * n2
    solve_fresh = solve_known + 160 * rows + 48 * n1
    relax = solve_fresh + 8 * n1
    prepare = 560 * rows + 256 * n1 + 8 * n2
    slipped = 289 * rows + 32 * n1
    body = copy.awake_count * (200 + SUBSTEPS * (124 + 300))
    total = prepare + SUBSTEPS * (warm + relax) + solve_fresh + (SUBSTEPS - 1) * solve_known + slipped + body
    return int(total)


def batch_algorithmic_bytes(batch):
    """algorithmic_bytes over every world of a batch (a BatchCopy): each world's solved rows are
    its first starts[33] rows, and every awake body of every world takes the body passes."""
    import numpy as np
    st = batch.stage
    pts = np.concatenate([st.rows["points"][int(batch.row_offset[w]): int(batch.row_offset[w]) + int(batch.starts[35 * w + 33])]
                          for w in range(batch.worlds)]).astype(np.int64)

    class Solved:
        rows = {"points": pts}
        solved = int(pts.size)
        awake_count = st.awake_count

    return algorithmic_bytes(Solved)


# ---- clocks -------------------------------------------------------------------------------

class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(s[1]) for s in self.samples if len(s) >= 9 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) >= 9 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples if len(s) >= 9 for k in range(4)
                          if s[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ---- timing -------------------------------------------------------------------------------

def time_resident(lib, ctx, copy, steps, warmup, torch):
    """bg_solve over the uploaded input: restore and flush untimed, events around the solve."""
    from bearing_b200 import _ffi
    B, R, S = copy.views()
    rc = lib.bg_upload(ctx, C.byref(B), C.byref(R))
    assert rc == 0, lib.bg_last_error(ctx)
    stream = torch.cuda.ExternalStream(lib.bg_stream(ctx))
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > L2
    times, stage, launches = [], [], 0
    for i in range(warmup + steps):
        assert lib.bg_restore(ctx) == 0
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        before = lib.bg_last_launches(ctx)
        torch.cuda.nvtx.range_push("timed" if i >= warmup else "warmup")
        e0.record(stream)
        rc = lib.bg_solve(ctx, C.byref(S))
        e1.record(stream)
        torch.cuda.nvtx.range_pop()
        assert rc == 0, lib.bg_last_error(ctx)
        e1.synchronize()
        if i >= warmup:
            times.append(e0.elapsed_time(e1))
            stage.append(lib.bg_last_stage_ms(ctx))
            launches += lib.bg_last_launches(ctx) - before
    # The result of the last timed solve, checked for completion (a lost step raises).
    out = copy.copy()
    Bo, Ro, _ = out.views()
    rc = lib.bg_download(ctx, C.byref(Bo), C.byref(Ro))
    assert rc == 0, lib.bg_last_error(ctx)
    return times, stage, launches, out


def host_views(work):
    """The views bg_solve_step gets from a World: every column, except the three written columns
    only slipped() reads after the stage (sliding, anchor_a, anchor_b), which it runs on the device
    itself; those are NULL and not copied back."""
    B, R, S = work.views()
    R.sliding = None
    R.anchor_a = None
    R.anchor_b = None
    return B, R, S


def time_e2e(lib, ctx, copy, steps, warmup, torch, host="page-locked"):
    """bg_solve_step end to end: uploads, solve and downloads inside the timed region.  `host` is
    where the caller's columns live: "page-locked" (allocated pinned, as a World that keeps its
    columns pinned passes them), "registered" (ordinary arrays, page-locked in place once by
    bg_register_host, as a World does when its columns are made or grow) or "pageable" (ordinary
    arrays).  The arrays are refilled with the step's input, untimed, before every call."""
    stream = torch.cuda.ExternalStream(lib.bg_stream(ctx))
    work = copy.pinned() if host == "page-locked" else copy.copy()
    if host == "registered":
        B, R, _ = host_views(work)
        rc = lib.bg_register_host(ctx, C.byref(B), C.byref(R), work.count)
        assert rc == 0, lib.bg_last_error(ctx)
    times = []
    for i in range(warmup + steps):
        work.fill(copy)
        B, R, S = host_views(work)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = lib.bg_solve_step(ctx, C.byref(B), C.byref(R), C.byref(S))
        e1.record(stream)
        assert rc == 0, lib.bg_last_error(ctx)
        e1.synchronize()
        if i >= warmup:
            times.append(e0.elapsed_time(e1))
    if host == "registered":
        assert lib.bg_unregister_host(ctx) == 0
    return times


def io_bytes(copy):
    """Bytes bg_solve_step copies in and out per step, from the columns it moves: every body and row
    column in (the output-only sliding and anchors excepted), and every written column out but the
    three host_views leaves NULL."""
    from stage_io import BODY_COLUMNS, ROW_COLUMNS, BODY_OUT, ROW_OUT
    h2d_row = [f for f, _, _ in ROW_COLUMNS if f not in ("sliding", "anchor_a", "anchor_b")]
    h2d = sum(copy.body[f].nbytes for f, _, _ in BODY_COLUMNS) + copy.awake_list.nbytes + \
        sum(copy.rows[f].nbytes for f in h2d_row)
    d2h = sum(copy.body[f].nbytes for f in BODY_OUT) + sum(copy.rows[f].nbytes for f in ROW_OUT)
    return int(h2d), int(d2h)


def cpu_solve_times(copy, workers, sample):
    """The CPU restatement of the reference's solve stage, timed on `sample` solve stages."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_io
    times = []
    for _ in range(sample):
        work = copy.copy()
        t0 = time.perf_counter()
        oracle_io.solve(work, workers)
        times.append(time.perf_counter() - t0)
    return times


def profiled(name):
    """One entry of profiles/counters.json (the ncu counters the bench's rooflines use), or None."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "counters.json")))[name]
    except (OSError, ValueError, KeyError):
        return None


def measured_traffic(bodies, at, algorithmic):
    """DRAM bytes per launch of the stage kernel, from the committed ncu capture of the same input
    (the pile's step 301); for another step of the same pile, scaled by the two launches'
    algorithmic bytes (the traffic grows with the rows and points a launch works through); None
    for another workload."""
    got = profiled("stage_grid_pile50k_step301")
    if bodies != 50_000 or got is None:
        return None, None
    if at == 300:
        return int(got["traffic_bytes_per_launch"]), "ncu capture of this launch (profiles/counters.json)"
    return int(round(got["traffic_bytes_per_launch"] * algorithmic / got["algorithmic_bytes_per_launch"])), \
        "ncu capture at step 301, scaled by algorithmic bytes"


def measure_batch(args, lib, torch, device, log, rank=0, world_size=1, dist=None):
    """Batched worlds: many small independent worlds solved in one launch (bg_batch_*: one CTA a
    world or all of them on the persistent grid, as the library's tuner picks), against the plain
    path called world by world (bg_solve_step).  The worlds (a pyramid, a box
    stack or a sphere pile of 8..512 bodies each, friction U(0.3, 0.8), restitution U(0, 0.4)) are
    stepped together to step `batch_at`; then that step's solve stage is timed: batched with its
    input resident, batched through bg_batch_solve_step with host arrays, and as a loop of
    bg_solve_step over the worlds (host arrays too).  The loop's results must equal the batch's
    bit for bit.  Under torchrun the worlds are sharded over the ranks by their body counts
    (bearing_b200.shard), each rank building and solving only its own; times are the max over
    ranks, and no data crosses between ranks."""
    from bearing_b200 import scenes, shard
    from bearing_b200.world import Batch, World
    from stage_io import BatchCopy, first_difference
    seed = 4096
    weights = [scenes.batch_world_bodies(seed, i) for i in range(args.batch_worlds)]
    mine = shard.shard_of(weights, rank, world_size)
    t0 = time.time()
    worlds = []
    for i in mine:
        w = World({}, solver=(0, 0))   # stepped by the batch, never by a solver of its own
        scenes.batch_world(w, scenes.batch_rng(seed, i))
        worlds.append(w)
    batch = Batch(worlds, device=device, threads=host_threads())
    for _ in range(args.batch_at):
        batch.step(DT)
    batch.begin_step(DT)
    base = BatchCopy(*batch.views())
    if args.save_batch:
        base.save(args.save_batch)
    if log:
        log(f"batch of {args.batch_worlds} worlds built and stepped to {args.batch_at} in {time.time() - t0:.0f} s: "
            f"{base.stage.capacity} slots, {base.stage.count} rows")
    ctx = lib.bg_create(device, 0)
    stream = torch.cuda.ExternalStream(lib.bg_stream(ctx))
    # resident
    B, R, W, S = base.views()
    assert lib.bg_batch_upload(ctx, C.byref(B), C.byref(R), C.byref(W)) == 0, lib.bg_last_error(ctx)
    resident = []
    for i in range(args.warmup + args.steps):
        assert lib.bg_restore(ctx) == 0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        assert lib.bg_batch_solve(ctx, C.byref(S)) == 0, lib.bg_last_error(ctx)
        e1.record(stream)
        e1.synchronize()
        if i >= args.warmup:
            resident.append(e0.elapsed_time(e1))
    cta_threads = lib.bg_block_threads(ctx)   # chosen by the library's tuner on the first solve
    split = None
    if world_size == 1:
        split = measure_batch_split(args, lib, torch, device, base, statistics.mean(resident), log)
    # batched, host arrays: pageable (as the loop below has them), then page-locked.  A large
    # batch moves in groups of worlds on contexts of the library's own, so the events only bracket
    # the synchronous call (the context's own stream is idle meanwhile).
    def batched_e2e(work):
        times = []
        for i in range(args.warmup + args.steps):
            work.fill(base)
            B, R, W, S = work.views()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            assert lib.bg_batch_solve_step(ctx, C.byref(B), C.byref(R), C.byref(W), C.byref(S)) == 0, lib.bg_last_error(ctx)
            e1.record(stream)
            e1.synchronize()
            if i >= args.warmup:
                times.append(e0.elapsed_time(e1))
        return times

    batched_locked = batched_e2e(base.pinned())
    work = base.copy()
    batched = batched_e2e(work)
    # the plain path, world by world: each world's solve stage with its input resident (uploaded
    # untimed, events around bg_solve), summed over the worlds
    parts = [base.world(i) for i in range(base.worlds)]
    one = lib.bg_create(device, 0)
    one_stream = torch.cuda.ExternalStream(lib.bg_stream(one))
    loop_resident = 0.0
    for p in parts:
        Bw, Rw, Sw = p.views()
        assert lib.bg_upload(one, C.byref(Bw), C.byref(Rw)) == 0, lib.bg_last_error(one)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(one_stream)
        assert lib.bg_solve(one, C.byref(Sw)) == 0, lib.bg_last_error(one)
        e1.record(one_stream)
        e1.synchronize()
        loop_resident += e0.elapsed_time(e1)
    loop = []
    for i in range(2):
        outs = [p.copy() for p in parts]
        views = [o.views() for o in outs]
        torch.cuda.synchronize()
        t = time.perf_counter()
        for Bw, Rw, Sw in views:
            assert lib.bg_solve_step(one, C.byref(Bw), C.byref(Rw), C.byref(Sw)) == 0, lib.bg_last_error(one)
        torch.cuda.synchronize()
        loop.append((time.perf_counter() - t) * 1000)
    same = all(first_difference(work.world(i), outs[i]) is None for i in range(base.worlds))
    lib.bg_destroy(one)
    lib.bg_destroy(ctx)
    batch.destroy()
    ms_res, ms_bat, ms_loop = statistics.mean(resident), statistics.mean(batched), min(loop)
    ms_lock = statistics.mean(batched_locked)
    ms_loop_res = loop_resident
    algo = batch_algorithmic_bytes(base)   # this rank's worlds
    slots, rows = int(base.stage.capacity), int(base.stage.count)
    solved = int(sum(int(base.starts[k * 35 + 33]) for k in range(base.worlds)))
    if dist:
        t = torch.tensor([ms_res, ms_bat, ms_loop, ms_lock, ms_loop_res], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_res, ms_bat, ms_loop, ms_lock, ms_loop_res = (float(x) for x in t.tolist())
        t = torch.tensor([slots, rows, solved, 0 if same else 1], device="cuda", dtype=torch.int64)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        slots, rows, solved, unequal = (int(x) for x in t.tolist())
        same = unequal == 0
    n = args.batch_worlds
    return {"workload": f"{n} independent worlds (pyramid, box stack or sphere pile of 8..512 bodies), "
                        f"solve stage at step {args.batch_at + 1}",
            "worlds": n, "ranks": world_size, "slots": slots, "rows": rows, "solved_rows": solved,
            "unit": "world-steps/s",
            "batched_resident": {"value": n / (ms_res / 1000), "ms_per_step": ms_res},
            "batched_e2e": {"value": n / (ms_bat / 1000), "ms_per_step": ms_bat, "host_memory": "pageable"},
            "batched_e2e_page_locked": {"value": n / (ms_lock / 1000), "ms_per_step": ms_lock},
            "per_world_loop_e2e": {"value": n / (ms_loop / 1000), "ms_per_step": ms_loop},
            "per_world_loop_resident": {"value": n / (ms_loop_res / 1000), "ms_per_step": ms_loop_res,
                                        "how": "sum over the worlds of bg_solve with that world's input resident"},
            "speedup_e2e": ms_loop / ms_bat, "speedup_resident": ms_loop_res / ms_res,
            "bit_identical": same, "cta_threads": cta_threads,
            "roofline": batch_roofline(algo, ms_res, cta_threads), "size_class_split": split}


def measure_batch_split(args, lib, torch, device, base, ms_whole, log):
    """The batch split by size class: its small worlds (at most `cut` solved rows) one CTA a world
    at a fixed CTA size, its large ones on the persistent grid, each half resident and timed on
    its own (the grid kernel holds every SM, so the halves run one after the other and the split
    costs their sum), against the whole batch as the tuner ran it; the best split's results are
    checked against the whole batch's, world by world."""
    import numpy as np
    from stage_io import first_difference
    solved = np.array([int(base.starts[k * 35 + 33]) for k in range(base.worlds)])

    def resident(sub, threads):
        ctx = lib.bg_create(device, 0)
        assert lib.bg_set_block_threads(ctx, threads) == 0
        stream = torch.cuda.ExternalStream(lib.bg_stream(ctx))
        B, R, W, S = sub.views()
        assert lib.bg_batch_upload(ctx, C.byref(B), C.byref(R), C.byref(W)) == 0, lib.bg_last_error(ctx)
        times = []
        for i in range(args.warmup + args.steps):
            assert lib.bg_restore(ctx) == 0
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            assert lib.bg_batch_solve(ctx, C.byref(S)) == 0, lib.bg_last_error(ctx)
            e1.record(stream)
            e1.synchronize()
            if i >= args.warmup:
                times.append(e0.elapsed_time(e1))
        out = sub.copy()
        Bo, Ro, _, _ = out.views()
        assert lib.bg_batch_download(ctx, C.byref(Bo), C.byref(Ro)) == 0
        lib.bg_destroy(ctx)
        return statistics.mean(times), out

    tried = []
    best = None
    for cut in (16, 64, 256):
        small = np.flatnonzero(solved <= cut)
        large = np.flatnonzero(solved > cut)
        if small.size == 0 or large.size == 0:
            continue
        sub_s, sub_l = base.subset(small), base.subset(large)
        ms_l, out_l = resident(sub_l, _ffi_grid())
        for threads in (64, 128):
            ms_s, out_s = resident(sub_s, threads)
            tried.append({"cut_rows": cut, "small_worlds": int(small.size), "cta_threads": threads,
                          "small_ms": ms_s, "large_ms": ms_l, "ms_per_step": ms_s + ms_l})
            if best is None or ms_s + ms_l < best[0]:
                best = (ms_s + ms_l, small, large, out_s, out_l)
    if best is None:
        return None
    # the whole batch's own results, solved once more as it ran
    whole = base.copy()
    ctx = lib.bg_create(device, 0)
    B, R, W, S = whole.views()
    assert lib.bg_batch_solve_step(ctx, C.byref(B), C.byref(R), C.byref(W), C.byref(S)) == 0
    lib.bg_destroy(ctx)
    _, small, large, out_s, out_l = best
    same = all(first_difference(whole.world(int(w)), out_s.world(j)) is None for j, w in enumerate(small)) and \
        all(first_difference(whole.world(int(w)), out_l.world(j)) is None for j, w in enumerate(large))
    result = {"what": "small worlds one CTA a world, large ones on the grid, run one after the other",
              "whole_batch_ms": ms_whole, "best_split_ms": best[0], "tried": tried, "bit_identical": same}
    if log:
        log(f"batch split by size class: best {best[0]:.2f} ms against {ms_whole:.2f} ms for the whole batch "
            f"as the tuner ran it; bit-identical {same}")
    return result


def _ffi_grid():
    from bearing_b200 import _ffi
    return _ffi.BG_BATCH_ON_GRID


def solve_saved_batch(args, log):
    """One batched solve of a saved batch on the persistent grid (no tuning), for a profiler."""
    from bearing_b200 import _ffi
    from stage_io import BatchCopy
    lib = _ffi.gpu()
    base = BatchCopy.load(args.load_batch)
    ctx = lib.bg_create(0, 0)
    assert lib.bg_set_block_threads(ctx, _ffi.BG_BATCH_ON_GRID) == 0
    B, R, W, S = base.views()
    assert lib.bg_batch_upload(ctx, C.byref(B), C.byref(R), C.byref(W)) == 0, lib.bg_last_error(ctx)
    assert lib.bg_batch_solve(ctx, C.byref(S)) == 0, lib.bg_last_error(ctx)
    ms = lib.bg_last_stage_ms(ctx)
    lib.bg_destroy(ctx)
    if log:
        log(f"saved batch: {base.worlds} worlds, {base.stage.count} rows, stage {ms:.3f} ms")


def measure_adjoint(args, device, log):
    """The differentiable workload: `adjoint_worlds` towers struck by a ball (scenes.tower), stepped
    `adjoint_steps` times as one batch with a checkpoint every 20 steps, then the backward pass: the
    gradient of each tower's loss with respect to its friction, restitution and launch velocity
    (bearing_b200.adjoint.tower_gradients).  Timed end to end on the host clock (the forward steps,
    then the backward pass: recomputing each 20-step segment, the host's reverse and bg_backward);
    the adjoint kernels' own device time beside it.  CPU baseline: the oracle's dual-number run of
    a sample of the same towers (five directions at once: one forward pass gives the same five
    derivatives), on one thread."""
    from bearing_b200 import adjoint, scenes
    from bearing_b200.world import World
    import numpy as np
    import oracle_io
    n, steps = args.adjoint_worlds, args.adjoint_steps
    t0 = time.perf_counter()
    out = adjoint.tower_gradients(n, seed=5000, steps=steps, checkpoint=20, device=device)
    wall = time.perf_counter() - t0
    if log:
        log(f"adjoint: {n} towers x {steps} steps: forward {out['forward_s']:.1f} s, backward "
            f"{out['backward_s']:.1f} s ({out['device_ms'] / 1000:.1f} s in the adjoint kernels)")
    sample = 2
    tc = time.perf_counter()
    worst = 0.0
    for i in range(sample):
        w = World({}, solver=oracle_io.solver(0))
        _, info = scenes.tower(w, scenes.batch_rng(5000, i))
        dual = oracle_io.DualWorld(w, info["friction"], info["restitution"], info["ball"])
        for _ in range(steps):
            dual.step(DT)
        g = np.zeros(5)
        for s, t in zip(info["cubes"], info["targets"]):
            v, tan = dual.pose(s)
            g += 2 * (v[:3] - t) @ tan[:3]
        dual.close()
        w.destroy()
        worst = max(worst, float(np.max(np.abs(out["gradients"][i] - g)) / np.max(np.abs(g))))
    cpu_s = (time.perf_counter() - tc) / sample
    return {"workload": f"{n} towers (3 x 10 cubes of 0.5 m) struck by a 50 kg ball, {steps} steps, "
                        f"checkpoint every 20 steps; gradients of each tower's loss w.r.t. friction, "
                        f"restitution and the launch velocity",
            "unit": "tower-gradients/s", "value": n / (out["forward_s"] + out["backward_s"]),
            "forward_s": out["forward_s"], "backward_s": out["backward_s"], "wall_s": wall,
            "adjoint_kernel_s": out["device_ms"] / 1000, "tape_peak_nodes": out["tape_peak"],
            "backward_parts_s": out["backward_parts"],
            "roofline": {"bound": "hbm", "kernel": "adjoint_step",
                         "achieved": out["device_bytes"] / (out["device_ms"] / 1000) / 1e9, "peak": hbm_peak()[0],
                         "unit": "GB/s", "frac": out["device_bytes"] / (out["device_ms"] / 1000) / 1e9 / hbm_peak()[0],
                         "algorithmic_bytes": out["device_bytes"],
                         "bytes_are": "each row's records, prepared terms and adjoints per pass, each body's per "
                                      "substep (bg_backward_bytes), over the adjoint kernels' device time"},
            "check": {"worlds": sample, "max_rel_err_vs_dual_numbers": worst},
            "cpu_baseline": {"value": 1 / cpu_s, "unit": "tower-gradients/s", "cores": 1, "kind": "port",
                             "sample": f"{sample} towers' dual-number runs (the oracle, 5 directions) on one "
                                       f"thread"}}


def measure_narrowphase(lib, ctx, world, steps, warmup, threads, log):
    """The narrowphase of the same step on the device: bg_collide over the pairs the step's own
    narrowphase handed to collide() (bw_narrow_pairs), with the world's bodies; the kernel's
    device time and the call end to end (pairs and body columns in, manifolds out, on the host
    clock), against the host's narrowphase over the same list on every host thread
    (bw_collide_pairs), and the two results compared bit for bit."""
    import numpy as np
    import narrow_io
    from bearing_b200 import _ffi
    pairs = narrow_io.world_pairs(world)
    B, _, S = world.views()
    g = np.asarray(S.gravity, np.float64)
    out = narrow_io.ManifoldSet(pairs.count)
    view = pairs.view()
    kernel, e2e = [], []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        rc = lib.bg_collide(ctx, C.byref(B), g.ctypes.data_as(C.POINTER(C.c_double)), C.byref(view), C.byref(out.s))
        t1 = time.perf_counter()
        assert rc == 0, lib.bg_last_error(ctx)
        if i >= warmup:
            e2e.append((t1 - t0) * 1000)
            kernel.append(lib.bg_last_collide_ms(ctx))
    cpu = []
    for _ in range(2):
        t0 = time.perf_counter()
        host = narrow_io.host_collide(B, tuple(S.gravity), pairs, threads=threads)
        cpu.append((time.perf_counter() - t0) * 1000)
    same = narrow_io.first_unequal(host, out) is None
    # The host side of one step (bounds, broadphase, narrowphase, emit, carry, colour), on copies of
    # the world: with the host's own narrowphase (one thread, as the step runs it), and with the
    # narrowphase handed to bg_collide (bw_set_narrowphase).
    h = _ffi.host()

    def host_side(fn, user):
        best = None
        for _ in range(3):
            clone = h.bw_clone(world._w)
            assert clone and h.bw_set_narrowphase(clone, fn, user) == 0
            t0 = time.perf_counter()
            rc = h.bw_begin_step(clone, DT)
            dt_ms = (time.perf_counter() - t0) * 1000
            h.bw_destroy(clone)
            assert rc == 0
            best = dt_ms if best is None else min(best, dt_ms)
        return best

    step_host = host_side(None, None)
    step_device = host_side(C.cast(lib.bg_collide, C.c_void_p).value, ctx)
    n = pairs.count
    counts = np.bincount(out.points[:n], minlength=5)
    in_bytes = n * (2 * 4 + 2 * 8) + B.capacity * (11 * 8 + 2)
    out_bytes = n * (1 + 3 * 8 + 12 * 8 + 4 * 8 + 4 * 4)
    k_ms, e_ms, c_ms = statistics.mean(kernel), statistics.mean(e2e), min(cpu)
    if log:
        log(f"narrowphase: {n} pairs, kernel {k_ms:.3f} ms, end to end {e_ms:.3f} ms, host {c_ms:.1f} ms "
            f"({threads} threads), bit-identical {same}; host side of a step {step_host:.1f} ms, "
            f"{step_device:.1f} ms with bg_collide")
    return {"workload": f"the pile's step-{world.stats()['step'] + 1} narrowphase: the pairs whose boxes meet",
            "pairs": n, "manifolds_by_points": [int(x) for x in counts], "unit": "pairs/s",
            "value": n / (k_ms / 1000), "kernel_ms": k_ms,
            "e2e": {"value": n / (e_ms / 1000), "ms_per_step": e_ms, "h2d_bytes_per_step": int(in_bytes),
                    "d2h_bytes_per_step": int(out_bytes)},
            "cpu_baseline": {"value": n / (c_ms / 1000), "unit": "pairs/s", "cores": threads, "kind": "port",
                             "ms": c_ms, "sample": "the same pair list through the host's narrowphase "
                                                   "(bw_collide_pairs), every host thread"},
            "bit_identical": same,
            "host_step_ms": {"host_narrowphase": step_host, "device_narrowphase": step_device,
                             "what": "the host side of one step of the pile (bounds, broadphase, narrowphase, emit, "
                                     "carry, colour), best of 3 on copies of the world"}}


def measure_colouring(lib, ctx, copy, steps, warmup, log):
    """The colouring of the same step on the device: bg_colour over the step's manifolds in found
    order (recovered from the rows' found-order map), its kernels' device time and the call end to
    end, against the host's colouring of the same list (bw_colour_rows, one thread, as the step runs
    it), and both against the step's own row order."""
    import numpy as np
    from bearing_b200 import _ffi
    n = copy.count
    row = copy.rows["row"][:n]
    a = np.ascontiguousarray(copy.rows["a"][row], np.int32)
    b = np.ascontiguousarray(copy.rows["b"][row], np.int32)
    B = _ffi.Bodies()
    B.capacity = copy.capacity
    B.type = copy.body["type"].ctypes.data_as(C.POINTER(C.c_uint8))
    B.frozen = copy.body["frozen"].ctypes.data_as(C.POINTER(C.c_uint8))
    pi = C.POINTER(C.c_int32)

    def arrays():
        return (np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(_ffi.BG_STARTS, np.int32), C.c_int32())

    def call(fn, *lead):
        colour, order, starts, solved = arrays()
        t0 = time.perf_counter()
        rc = fn(*lead, C.byref(B), n, a.ctypes.data_as(pi), b.ctypes.data_as(pi), colour.ctypes.data_as(pi),
                order.ctypes.data_as(pi), starts.ctypes.data_as(pi), C.byref(solved))
        ms = (time.perf_counter() - t0) * 1000
        assert rc == 0
        return ms, order, starts

    kernel, e2e = [], []
    for i in range(warmup + steps):
        ms, order, starts = call(lib.bg_colour, ctx)
        if i >= warmup:
            e2e.append(ms)
            kernel.append(lib.bg_last_colour_ms(ctx))
    host = _ffi.host()
    cpu = [call(host.bw_colour_rows)[0] for _ in range(3)]
    _, horder, hstarts = call(host.bw_colour_rows)
    found = np.empty(n, np.int32)
    found[row] = np.arange(n, dtype=np.int32)
    same = bool(np.array_equal(order, found) and np.array_equal(horder, found) and
                np.array_equal(starts, copy.starts) and np.array_equal(hstarts, copy.starts))
    k_ms, e_ms, c_ms = statistics.mean(kernel), statistics.mean(e2e), min(cpu)
    if log:
        log(f"colouring: {n} manifolds, kernels {k_ms:.3f} ms, end to end {e_ms:.3f} ms, host {c_ms:.2f} ms, "
            f"the step's own order {same}")
    return {"workload": "the pile's step-301 manifolds in found order: colours, row order and colour starts",
            "manifolds": n, "unit": "manifolds/s", "value": n / (k_ms / 1000), "kernel_ms": k_ms,
            "e2e": {"value": n / (e_ms / 1000), "ms_per_step": e_ms, "h2d_bytes_per_step": 8 * n + 2 * copy.capacity,
                    "d2h_bytes_per_step": 8 * n + 4 * 35},
            "cpu_baseline": {"value": n / (c_ms / 1000), "unit": "manifolds/s", "cores": 1, "kind": "port", "ms": c_ms,
                             "sample": "the same list through the host's colouring (bw_colour_rows)"},
            "same_as_the_step": same}


def measure_contact_step(args, lib, solver, world, device, steps, warmup, log):
    """A World step with its whole contact side on the device (bg_contact_step: narrowphase, rows,
    warm start, colouring, order, solve stage and store, the rows never on the host) against the same
    World step on the host path (the host's emit, carry, colour and keep around bg_collide and
    bg_solve_step), at the same steps of the same pile.  A second world is built in contact mode and
    stepped to the headline step; `world` (the headline's, begun at that step) finishes its step with
    bg_solve_step; both then take the same timed steps, their row counts compared at each."""
    from bearing_b200 import _ffi, scenes
    from bearing_b200.world import GpuSolver, World
    B, R, S = world.views()
    assert lib.bg_solve_step(solver.ctx, C.byref(B), C.byref(R), C.byref(S)) == 0
    world.end_step()
    dev = GpuSolver(device)
    wb = World({}, solver=dev)
    calls = []
    proto = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.POINTER(_ffi.Bodies), C.POINTER(_ffi.Materials),
                        C.POINTER(_ffi.ContactPairs), C.POINTER(_ffi.Step), C.POINTER(_ffi.ContactResult))

    def timed(user, bodies, materials, pairs, step, out):   # bg_contact_step, timed on the host clock
        t0 = time.perf_counter()
        rc = lib.bg_contact_step(user, bodies, materials, pairs, step, out)
        calls.append(((time.perf_counter() - t0) * 1000, pairs.contents.list.count, bodies.contents.capacity,
                      out.contents.rows))
        return rc
    hook = proto(timed)
    assert wb._lib.bw_set_contact_step(wb._w, C.cast(hook, C.c_void_p), C.c_void_p(dev.ctx)) == 0
    scenes.pile(wb, count=args.bodies, seed=50_000)
    t0 = time.time()
    for _ in range(args.at + 1):
        wb.step(DT)
    if log:
        log(f"contact-mode pile stepped to {args.at + 1} in {time.time() - t0:.0f} s: {wb.stats()}")
    same = wb.stats() == world.stats()
    host_ms, dev_ms, call_ms, parts = [], [], [], []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        world.step(DT)
        t1 = time.perf_counter()
        wb.step(DT)
        t2 = time.perf_counter()
        same = same and wb.stats() == world.stats()
        if i >= warmup:
            host_ms.append((t1 - t0) * 1000)
            dev_ms.append((t2 - t1) * 1000)
            call_ms.append(calls[-1][0])
            parts.append(dev.contact_ms())
    np_, nb, rows = calls[-1][1], calls[-1][2], calls[-1][3]
    # in: 43 FP64 body columns, 6 byte columns, joint_head, the awake list and 3 materials a slot, and the
    # pair list (a, b, memory, margin, tolerance); out: the 30 FP64 body columns the step writes, and each
    # pair's point count and touching flag
    h2d = nb * (43 * 8 + 6 + 4 + 4 + 3 * 8) + np_ * (3 * 4 + 2 * 8)
    d2h = nb * (30 * 8) + 2 * np_
    part = [statistics.mean(p[k] for p in parts) for k in range(4)]
    out = {"workload": f"World.step of the {args.bodies}-body pile at steps {args.at + 2 + warmup}.."
                       f"{args.at + 1 + warmup + steps}, its contact side on the device",
           "unit": "ms", "pairs_listed": np_, "rows": rows,
           "world_step_ms": statistics.mean(dev_ms), "host_path_world_step_ms": statistics.mean(host_ms),
           "contact_call_ms": statistics.mean(call_ms),
           "device_ms": {"narrowphase": part[0], "rows_colours_order": part[1], "solve_stage": part[2],
                         "store": part[3]},
           "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
           "same_counts_as_host_path": same,
           "what": "world_step_ms: World.step (host bounds, broadphase and pair upkeep, then bg_contact_step); "
                   "host_path_world_step_ms: World.step with the host's rows (bg_collide narrowphase, host emit/carry/"
                   "colour/arrange, bg_solve_step with pageable columns, host keep); contact_call_ms: bg_contact_step "
                   "end to end on the host clock (bodies and pair list in, bodies out)"}
    if log:
        log(f"contact step: World.step {out['world_step_ms']:.1f} ms against {out['host_path_world_step_ms']:.1f} ms "
            f"on the host path; bg_contact_step {out['contact_call_ms']:.2f} ms ({np_} pairs, {rows} rows; device "
            f"{part[0]:.3f} + {part[1]:.3f} + {part[2]:.3f} + {part[3]:.3f} ms); same counts {same}")
    wb.destroy()
    dev.close()
    return out


def batch_roofline(algo, ms, cta_threads):
    """The batched kernel's roofline line: this rank's algorithmic bytes over the resident solve's
    time (the max over ranks), against the measured HBM copy rate; DRAM traffic from the committed
    capture of the same 4,096 worlds at step 301, scaled by algorithmic bytes where the batch differs."""
    hbm, peak_source = hbm_peak()
    achieved = algo / (ms / 1000) / 1e9
    traffic, source = None, None
    got = profiled("stage_grid_batch_4096worlds_step301")
    if got is not None and cta_threads == 1:   # the capture is of the grid's kernel
        traffic = int(round(got["traffic_bytes_per_launch"] * algo / got["algorithmic_bytes_per_launch"]))
        source = ("ncu capture of this launch (profiles/counters.json)" if algo == got["algorithmic_bytes_per_launch"]
                  else "ncu capture of the 4,096 worlds at step 301, scaled by algorithmic bytes")
    kernel = "stage_grid_batch" if cta_threads == 1 else f"stage_block ({cta_threads} threads a world)"
    return {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "algorithmic_bytes": algo, "traffic": traffic, "traffic_source": source,
            "peak_source": peak_source}


def hbm_peak():
    """The HBM denominator: the measured copy rate in MEASURED_PEAKS.json where that file exists,
    else the earlier measurement of this GPU type's copy rate, 6,650 GB/s."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), \
            "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except (OSError, ValueError, KeyError):
        return 6650.0, "6,650 GB/s, an earlier copy-rate measurement on B200 (of fallback; no MEASURED_PEAKS.json)"


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---- main ---------------------------------------------------------------------------------

def main():
    args = parse()
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    log = (lambda s: print(f"[bench] {s}", file=sys.stderr, flush=True)) if rank == 0 else None

    config = {"workload": f"{args.bodies}-body mixed pile (60% boxes, 25% spheres, 15% capsules), solve stage "
                          f"at step {args.at + 1}", "bodies": args.bodies, "at_step": args.at + 1,
              "substeps": SUBSTEPS, "dt": DT, "l2": "flushed between timed iterations (256 MB write)",
              "parallelism": f"replicas x{args.gpus}"}

    if args.impl == "reference":
        if rank != 0:
            return
        from stage_io import StageCopy
        import oracle_io
        threads = host_threads()
        workers = max(0, threads - 1)
        w = build_pile(oracle_io.solver(workers), args.bodies, args.at, log)
        copy = StageCopy(w)
        rows_per_stage = copy.solved * SUBSTEPS * 3
        cpu_solve_times(copy, workers, 1)
        times = []
        for _ in range(args.warmup):
            cpu_solve_times(copy, workers, 1)
        for _ in range(args.steps):
            times += cpu_solve_times(copy, workers, 1)
        sec = statistics.mean(times)
        value = rows_per_stage / sec
        line = {"metric": "contact rows/s", "value": value, "unit": "rows/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1000, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
                "impl": "reference", "config": dict(config, rows=copy.solved, cpu_threads=threads),
                "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "port",
                                 "sample": f"{args.steps} solve stages of the step-{args.at + 1} input, "
                                           f"{workers} workers + the calling thread (src/core/jobs.js split)"},
                "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    if args.load_batch:
        solve_saved_batch(args, log)
        return
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world_size > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    from bearing_b200 import _ffi
    from bearing_b200.world import GpuSolver
    from stage_io import StageCopy
    lib = _ffi.gpu()
    solver = GpuSolver(local)
    t0 = time.time()
    w = None
    if args.load_input:
        copy = StageCopy.load(args.load_input)
    else:
        w = build_pile(solver, args.bodies, args.at, log)
        if log:
            log(f"pile built to step {args.at} in {time.time() - t0:.0f} s: {w.stats()}")
        copy = StageCopy(w)
        if args.save_input:
            copy.save(args.save_input)
    ctx = lib.bg_create(local, 0)
    assert ctx, "bg_create failed"
    h2d, d2h = io_bytes(copy)
    algo = algorithmic_bytes(copy)
    clocks = Clocks(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    times, stage, launches, out = time_resident(lib, ctx, copy, args.steps, args.warmup, torch)
    clock = clocks.stop()
    e2e_times = times if args.resident_only else time_e2e(lib, ctx, copy, args.steps, args.warmup, torch)
    pageable_times = times if args.resident_only else time_e2e(lib, ctx, copy, args.steps, args.warmup, torch,
                                                                host="pageable")
    registered_times = times if args.resident_only else time_e2e(lib, ctx, copy, args.steps, args.warmup, torch,
                                                                  host="registered")
    torch.cuda.synchronize()
    ms = statistics.mean(times)
    ms_e2e = statistics.mean(e2e_times)
    ms_pageable = statistics.mean(pageable_times)
    ms_registered = statistics.mean(registered_times)
    ms_stage = statistics.mean(stage)
    if dist:
        t = torch.tensor([ms, ms_e2e, ms_stage, ms_pageable, ms_registered], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_e2e, ms_stage, ms_pageable, ms_registered = (float(x) for x in t.tolist())
    rows_per_stage = copy.solved * SUBSTEPS * 3
    value = world_size * rows_per_stage / (ms / 1000)
    e2e = world_size * rows_per_stage / (ms_e2e / 1000)
    hbm, peak_source = hbm_peak()
    achieved = algo / (ms_stage / 1000) / 1e9
    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu and not args.resident_only:
        threads = host_threads()
        t1 = cpu_solve_times(copy, 0, args.cpu_sample)
        cpu = {"value": rows_per_stage / statistics.mean(t1), "unit": "rows/s", "cores": 1, "kind": "port",
               "sample": f"{args.cpu_sample} solve stages of the step-{args.at + 1} input "
                         f"({copy.solved} rows), 1 thread",
               "threads_available": threads}
        if threads > 1:
            tn = cpu_solve_times(copy, threads - 1, args.cpu_sample)
            cpu["all_threads"] = {"value": rows_per_stage / statistics.mean(tn), "cores": threads}
    batch = None
    if not args.no_batch and not args.resident_only:   # every rank, or none: it holds collectives
        batch = measure_batch(args, lib, torch, local, log, rank, world_size, dist)
    narrow = None
    if not args.resident_only and rank == 0 and w is not None:
        narrow = measure_narrowphase(lib, ctx, w, args.steps, args.warmup, host_threads(), log)
    colouring = None
    if not args.resident_only and rank == 0:
        colouring = measure_colouring(lib, ctx, copy, args.steps, args.warmup, log)
    contact = None
    if not args.resident_only and rank == 0 and w is not None and not args.no_contact:
        contact = measure_contact_step(args, lib, solver, w, local, args.steps, max(3, args.warmup), log)
    adj = None
    if not args.no_adjoint and not args.resident_only and rank == 0 and world_size == 1:
        adj = measure_adjoint(args, local, log)
    traffic, traffic_source = measured_traffic(args.bodies, args.at, algo)
    if rank == 0:
        line = {"metric": "contact rows/s", "value": value, "unit": "rows/s", "n_gpus": world_size,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
                "config": dict(config, rows=copy.solved, points=int(copy.rows["points"][:copy.solved].sum()),
                               colours=int(sum(1 for k in range(32) if copy.starts[k + 1] > copy.starts[k])),
                               overflow=int(copy.starts[33] - copy.starts[32]), awake=copy.awake_count),
                "e2e": {"value": e2e, "unit": "rows/s", "ms_per_step": ms_e2e, "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "host_memory": "page-locked"},
                "e2e_pageable": {"value": world_size * rows_per_stage / (ms_pageable / 1000), "unit": "rows/s",
                                 "ms_per_step": ms_pageable, "host_memory": "pageable (ordinary numpy arrays)"},
                "e2e_registered": {"value": world_size * rows_per_stage / (ms_registered / 1000), "unit": "rows/s",
                                   "ms_per_step": ms_registered,
                                   "host_memory": "ordinary numpy arrays page-locked in place once by bg_register_host"},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                             "frac": achieved / hbm, "traffic": traffic, "traffic_source": traffic_source,
                             "kernel_ms": ms_stage,
                             "algorithmic_bytes": algo, "peak_source": peak_source},
                "cpu_baseline": cpu, "clocks": clock, "gpu_launches": launches, "batch": batch, "adjoint": adj,
                "narrowphase": narrow, "colouring": colouring, "contact_step": contact}
        print(json.dumps(line), flush=True)
    lib.bg_destroy(ctx)
    solver.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
