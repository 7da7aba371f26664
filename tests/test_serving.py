"""Serving loop: chunks of many samples submitted concurrently, continuously
batched on the device.  Every chunk's records must be exactly what the
chunk gets aligned alone (and what the oracle gives), and the per-sample
counters kept on the device must add up to the alone results."""
import threading
import time

import numpy as np
import pytest

from hera_b200 import workloads

pytestmark = pytest.mark.gpu


def _chunks(config1):
    """(sample, r1, r2) chunks of three read models and uneven sizes."""
    ann, tx, _ = config1
    out = []
    sizes = [3000, 11000, 700, 5000, 16000, 1, 2500, 9000]
    models = ["config1", "config3", "config4"]
    for k, n in enumerate(sizes):
        r1, r2 = workloads.pairs(models[k % 3], ann, tx, n, seed=200 + k)
        out.append((k % 5, r1, r2))
    return out


@pytest.mark.parametrize("borrow", [False, True])
def test_mix_equals_alone_and_oracle(config1, oracle1, borrow):
    """borrow: submit keeps the caller's read pointers (no copy); the reads
    stay alive here until every wait has returned."""
    if not __import__("torch").cuda.is_available():
        pytest.skip("no CUDA device")
    from hera_b200 import api
    chunks = _chunks(config1)
    ctx = api.Context(config1[2])
    try:
        alone = [ctx.align_pairs(r1, r2, 1) for _, r1, r2 in chunks]
        # a small batch size, so batches span chunks and chunks span batches
        srv = api.Server(ctx, batch_pairs=4096, max_slots=3, write_bam=1, max_samples=8, borrow_reads=borrow)
        tickets = [None] * len(chunks)

        def feed(ks):
            for k in ks:
                s, r1, r2 = chunks[k]
                tickets[k] = srv.submit(s, r1, r2)
                time.sleep(0.002)   # arrivals while earlier chunks run

        th = [threading.Thread(target=feed, args=(range(i, len(chunks), 2),)) for i in range(2)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        infos = []
        for k, (s, r1, r2) in enumerate(chunks):
            res, info = srv.wait(tickets[k])
            infos.append(info)
            ga, gm = alone[k].canonical(), res.canonical()
            assert ga == gm, f"chunk {k}: served records differ from the chunk aligned alone"
            assert info["n"] == r1.n and info["sample"] == s
            assert info["submit_ms"] <= info["admit_ms"] <= info["done_ms"]
        # the oracle on the served results of two chunk types
        for k in (1, 2):
            _, r1, r2 = chunks[k]
            assert alone[k].canonical() == oracle1.align_pairs(r1.copy(), r2.copy(), 1).canonical()
        st = srv.stats()
        assert st["chunks_done"] == len(chunks)
        assert st["pairs_done"] == sum(r1.n for _, r1, _ in chunks)
        assert st["slots"] >= 1 and 0 < st["p50_ms"] <= st["p99_ms"]
        # continuous batching: some chunk was spread over several batches and
        # some batch carried pieces of several chunks
        assert max(i["batches"] for i in infos) > 1
        assert st["batches"] < sum(i["batches"] for i in infos)
        # per-sample device state against the alone results
        want = {}
        for k, (s, _, _) in enumerate(chunks):
            t = api.tally(alone[k])
            acc = want.setdefault(s, {key: 0 for key in t})
            for key, v in t.items():
                acc[key] += v
        for s in range(8):
            got = srv.sample_stats(s)
            assert got == want.get(s, {key: 0 for key in got}), f"sample {s}"
        srv.close()
    finally:
        ctx.close()


def test_server_rejects_bad_sample(config1):
    if not __import__("torch").cuda.is_available():
        pytest.skip("no CUDA device")
    from hera_b200 import api
    ann, tx, ix = config1
    ctx = api.Context(ix)
    try:
        srv = api.Server(ctx, batch_pairs=1024, max_slots=1, max_samples=4)
        r1, r2 = workloads.pairs("config1", ann, tx, 10, seed=5)
        with pytest.raises(api.HeraGpuError):
            srv.submit(4, r1, r2)
        t = srv.submit(3, r1, r2)
        res, info = srv.wait(t)
        assert res.recs.shape[0] == 20 and info["batches"] == 1
        srv.close()
    finally:
        ctx.close()


# ---- failures met on the host: nothing here faults a GPU ------------------

def test_server_creation_without_room_is_enomem(config1):
    """A reserve above the free device memory leaves no room for a batch
    slot: creation fails with HERA_GPU_ENOMEM and the context stays usable."""
    if not __import__("torch").cuda.is_available():
        pytest.skip("no CUDA device")
    from hera_b200 import api
    ann, tx, ix = config1
    ctx = api.Context(ix)
    try:
        with pytest.raises(api.HeraGpuError) as e:
            api.Server(ctx, batch_pairs=4096, hbm_reserve=1 << 50)
        assert e.value.code == -3
        r1, r2 = workloads.pairs("config1", ann, tx, 200, seed=6)
        assert ctx.align_pairs(r1, r2, 1).recs.shape[0] == 400
    finally:
        ctx.close()


def test_cancel_drops_one_sample_only(config1):
    """A sample cancelled while its chunks wait in the queue: its chunks not
    yet admitted end with HERA_GPU_ECANCELED, and every other sample's
    chunks come back exactly as aligned alone."""
    if not __import__("torch").cuda.is_available():
        pytest.skip("no CUDA device")
    from hera_b200 import api
    ann, tx, ix = config1
    ctx = api.Context(ix)
    try:
        chunks = []
        for k in range(12):
            r1, r2 = workloads.pairs("config1", ann, tx, 6000, seed=300 + k)
            chunks.append((k % 3, r1, r2))
        alone = [ctx.align_pairs(r1, r2, 1).canonical() for _, r1, r2 in chunks]
        # one slot and small batches: most of the plan waits in the queue
        srv = api.Server(ctx, batch_pairs=1024, max_slots=1, write_bam=1, max_samples=4)
        tickets = [srv.submit(s, r1, r2) for s, r1, r2 in chunks]
        n = srv.cancel(1)
        assert n >= 1
        cancelled = 0
        for k, (s, r1, r2) in enumerate(chunks):
            if s == 1:
                try:
                    res, _ = srv.wait(tickets[k])
                    assert res.canonical() == alone[k]   # admitted before the cancel
                except api.HeraGpuError as e:
                    assert e.code == api.HERA_GPU_ECANCELED
                    cancelled += 1
            else:
                res, _ = srv.wait(tickets[k])
                assert res.canonical() == alone[k], f"chunk {k} of sample {s}"
        assert cancelled == n
        # the sample can submit again
        t = srv.submit(1, chunks[1][1], chunks[1][2])
        assert srv.wait(t)[0].canonical() == alone[1]
        srv.close()
    finally:
        ctx.close()


def test_bad_chunk_in_a_mix_fails_alone(config1):
    """A chunk with a read longer than HERA_GPU_MAX_READ, submitted between
    others, is refused at submit with HERA_GPU_EINVAL; the chunks around it
    are served as if it had never come."""
    if not __import__("torch").cuda.is_available():
        pytest.skip("no CUDA device")
    from hera_b200 import api, synth
    ann, tx, ix = config1
    ctx = api.Context(ix)
    try:
        good = [workloads.pairs("config1", ann, tx, 3000, seed=400 + k) for k in range(4)]
        alone = [ctx.align_pairs(r1, r2, 1).canonical() for r1, r2 in good]
        b1, b2 = synth.simulate_pairs(tx, 50, seed=410, read_len=api.MAX_READ + 40)
        srv = api.Server(ctx, batch_pairs=2048, max_slots=2, write_bam=1, max_samples=4)
        tickets = [srv.submit(0, *good[0]), srv.submit(1, *good[1])]
        with pytest.raises(api.HeraGpuError) as e:
            srv.submit(2, b1, b2)
        assert e.value.code == -4
        tickets += [srv.submit(2, *good[2]), srv.submit(3, *good[3])]
        for k, t in enumerate(tickets):
            assert srv.wait(t)[0].canonical() == alone[k]
        srv.close()
    finally:
        ctx.close()
