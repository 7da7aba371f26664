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


def _small_index():
    from hera_b200 import index, synth
    ann = synth.make_annotation(seed=11, genome_len=300_000, n_genes=30, n_transcripts=75)
    tx = synth.transcriptome(ann)
    return ann, tx, index.build_index(tx)


def _chunk_classes(orc, ann, tx, cid):
    """The class table of chunk `cid` aligned alone (the oracle's records)."""
    from hera_b200 import workloads
    r1, r2 = workloads.pairs("config1" if cid % 2 else "config4", ann, tx, 1500 + 300 * cid, seed=400 + cid)
    return orc.classes([orc.align_pairs(r1, r2, 1)]), (r1, r2)


def test_class_tables_merge_equals_one_pass():
    """Per-chunk tables merged in chunk order == add_class over all chunks."""
    import oracle
    if not os.path.exists(oracle.ORACLE_SO):
        pytest.skip("oracle not built")
    ann, tx, ix = _small_index()
    orc = oracle.Oracle(ix)
    per, results = [], []
    for cid in range(5):
        t, (r1, r2) = _chunk_classes(orc, ann, tx, cid)
        per.append(t)
        results.append(orc.align_pairs(r1, r2, 1))
    whole = orc.classes(results)
    assert whole.n_classes > max(t.n_classes for t in per)
    assert shard.merge_class_tables(per).key() == whole.key()


def _class_worker(rank, world, port, q):
    import torch.distributed as dist
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ann, tx, ix = _small_index()
        orc = oracle.Oracle(ix)
        n = 5
        local = {cid: _chunk_classes(orc, ann, tx, cid)[0] for cid in shard.chunk_ids(n, rank, world)}
        merged = shard.gather_in_order(local, n)
        if rank == 0:
            q.put(shard.merge_class_tables(merged).key())
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_class_tables():
    """Two ranks build the class tables of their own chunks; rank 0 merges
    them in chunk order into the one-pass table."""
    import oracle
    if not os.path.exists(oracle.ORACLE_SO):
        pytest.skip("oracle not built")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_class_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ann, tx, ix = _small_index()
    orc = oracle.Oracle(ix)
    results = []
    for cid in range(5):
        _, (r1, r2) = _chunk_classes(orc, ann, tx, cid)
        results.append(orc.align_pairs(r1, r2, 1))
    assert got == orc.classes(results).key()


def test_class_table_merge_edges():
    """Chunks without classes, repeated ids keeping the first list, and
    PAIRED wrapping like hera's unsigned int."""
    import numpy as np
    from hera_b200.api import ClassTable

    def table(ids, counts, lists, tx, paired, frag):
        ns = np.array([len(x) for x in lists], np.uint32)
        off = np.zeros(len(ns), np.uint64)
        off[1:] = np.cumsum(ns[:-1])
        ref = np.concatenate([np.array(x, np.uint32) for x in lists]) if lists else np.zeros(0, np.uint32)
        return ClassTable(np.array(ids, np.uint32), np.array(counts, np.float64), ns, off, ref,
                          np.array(tx, np.uint32), paired, frag)

    a = table([7, 3], [2, 1], [[1, 2], [0, 3]], [1, 0, 0, 0], 0xFFFFFFFF, 10.0)
    empty = table([], [], [], [0, 2, 0, 0], 3, 4.0)
    b = table([9, 7], [5, 4], [[2, 3], [0, 1, 2]], [0, 0, 1, 0], 2, 1.0)
    m = shard.merge_class_tables([a, empty, b])
    assert m.ids.tolist() == [7, 3, 9]
    assert m.counts.tolist() == [6.0, 1.0, 5.0]
    assert m.lists() == [(1, 2), (0, 3), (2, 3)]   # id 7 keeps its first list
    assert m.tx_count.tolist() == [1, 2, 1, 0]
    assert m.paired == (0xFFFFFFFF + 3 + 2) & 0xFFFFFFFF
    assert m.mean_frag == 15.0
    with pytest.raises(ValueError):
        shard.merge_class_tables([])
