"""The multi-GPU (replica) split on CPU with gloo, world size 2: chunks are
dealt round robin, results merge back in chunk order, timings reduce by max."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from hera_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_chunk_ids_cover_once():
    for world in (1, 2, 3, 8):
        ids = sorted(i for r in range(world) for i in shard.chunk_ids(10, r, world))
        assert ids == list(range(10))


def test_merge_rejects_gaps_and_duplicates():
    with pytest.raises(ValueError):
        shard.merge_in_order([{0: "a"}, {0: "b"}], 1)
    with pytest.raises(ValueError):
        shard.merge_in_order([{0: "a"}], 2)


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 7
        local = {cid: f"chunk{cid}:rank{rank}" for cid in shard.chunk_ids(n, rank, world)}
        merged = shard.gather_in_order(local, n)
        t = shard.max_over_ranks(1.0 + rank)
        if rank == 0:
            q.put((merged, t))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged, t = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert merged == [f"chunk{i}:rank{i % 2}" for i in range(7)]
    assert t == 2.0
