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


def test_mix_equals_alone_and_oracle(config1, oracle1):
    if not __import__("torch").cuda.is_available():
        pytest.skip("no CUDA device")
    from hera_b200 import api
    chunks = _chunks(config1)
    ctx = api.Context(config1[2])
    try:
        alone = [ctx.align_pairs(r1, r2, 1) for _, r1, r2 in chunks]
        # a small batch size, so batches span chunks and chunks span batches
        srv = api.Server(ctx, batch_pairs=4096, max_slots=3, write_bam=1, max_samples=8)
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
