"""Independent worlds across ranks (bearing_b200.shard): the partition, and two ranks each stepping
only their own worlds reproduce one process stepping all of them, bit for bit.  The ranks are gloo
processes on the CPU with the oracle as each world's solve stage; on GPUs each rank would run its
shard with bg_batch_solve_step on its own device, which changes nothing about which worlds it owns."""
import hashlib
import multiprocessing as mp
import os
import socket

import pytest

from bearing_b200 import scenes, shard

SEED = 77
WORLDS = 14
STEPS = 12
DT = 1 / 60


def test_balance_covers_every_world_once_and_keeps_order():
    weights = [scenes.batch_world_bodies(SEED, i) for i in range(200)]
    for parts in (1, 2, 3, 8):
        shards = shard.balance(weights, parts)
        assert len(shards) == parts
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(200))
        for s in shards:
            assert s == sorted(s)
        loads = [sum(weights[i] for i in s) for s in shards]
        # the longest-processing-time rule: no rank above 4/3 of the best possible split
        assert max(loads) <= 4 / 3 * max(sum(weights) / parts, max(weights)) + 1e-9
    assert shard.shard_of(weights, 1, 2) == shard.balance(weights, 2)[1]
    with pytest.raises(ValueError):
        shard.shard_of(weights, 2, 2)


def fingerprints(indices):
    """Each world's FP64 state after STEPS steps with the oracle, as a digest."""
    import oracle_io
    from bearing_b200.world import World
    out = {}
    for i in indices:
        w = World({}, solver=oracle_io.solver(0))
        scenes.batch_world(w, scenes.batch_rng(SEED, i))
        for _ in range(STEPS):
            w.step(DT)
        st = w.state()
        out[i] = hashlib.sha256(b"".join(st[k].tobytes() for k in sorted(st))).hexdigest()
        w.destroy()
    return out


def _rank(rank, size, port, queue):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        weights = [scenes.batch_world_bodies(SEED, i) for i in range(WORLDS)]
        mine = shard.shard_of(weights, rank, size)
        got = [None] * size
        dist.all_gather_object(got, {"worlds": mine, "prints": fingerprints(mine)})
        if rank == 0:
            queue.put(got)
    finally:
        dist.destroy_process_group()


def test_two_ranks_step_their_shards_like_one_process():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    got = queue.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    owned = [i for g in got for i in g["worlds"]]
    assert sorted(owned) == list(range(WORLDS))
    assert all(g["worlds"] for g in got)
    merged = {i: h for g in got for i, h in g["prints"].items()}
    assert merged == fingerprints(range(WORLDS))
