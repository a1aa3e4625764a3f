"""Ensemble sharding over ranks (cryo_shard): the longest-processing-time
partition and the end-of-run gather, on CPU with gloo (world size 2)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import cryo_shard


def test_lpt_partition_properties():
    sizes = [5000, 200000, 12000, 150000, 7000, 7000, 90000, 64000, 31000]
    for world in (1, 2, 3, 4, 16):
        sh = cryo_shard.lpt_shards(sizes, world)
        assert len(sh) == world
        flat = sorted(t for s in sh for t in s)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[t] for t in s) for s in sh]
        if world <= len(sizes):
            # LPT: no rank exceeds the mean load by more than one tank
            assert max(loads) <= sum(sizes) / world + max(sizes)
    assert cryo_shard.lpt_shards([3, 1, 2], 2) == [[0], [2, 1]]
    with pytest.raises(ValueError):
        cryo_shard.lpt_shards([1], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, sizes, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        mine = cryo_shard.shard_of(sizes, rank, world)
        local = {t: {"rank": rank, "value": sizes[t] * 2} for t in mine}
        merged = cryo_shard.gather_per_tank(local)
        q.put((rank, sorted(merged), {t: v["value"] for t, v in merged.items()}))
    finally:
        dist.destroy_process_group()


def test_two_ranks_cover_every_tank_once():
    sizes = [5000, 200000, 12000, 150000, 7000, 90000, 64000]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, keys, vals in got:
        assert keys == list(range(len(sizes)))
        assert vals == {t: 2 * s for t, s in enumerate(sizes)}


def test_gather_without_process_group_is_local():
    assert cryo_shard.gather_per_tank({3: "x"}) == {3: "x"}
