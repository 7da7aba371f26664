"""Equivalence classes on the device (hera_gpu_classes_*): the add_class calls
of hera's host tail (src/hash_align.c:1564-1602) over the records, checked
against the reference's class goldens and against the oracle's restatement
on the config-1/config-4 read models, in one batch and in several."""
import json
import os

import numpy as np
import pytest

import oracle
from hera_b200 import api, index, synth, workloads

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SETS = ["pairs100", "pairs150div", "pairs_mixed", "pairs_long", "pairs_n", "single"]


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _to_device(torch, recs, pos, p):
    d_recs = torch.from_numpy(np.frombuffer(recs.tobytes(), np.uint8).copy()).cuda()
    d_pos = torch.from_numpy(np.ascontiguousarray(pos).view(np.int32).copy()).cuda()
    d_p = torch.from_numpy(np.ascontiguousarray(p, dtype=np.int32).copy()).cuda()
    torch.cuda.synchronize()
    return d_recs, d_pos, d_p


def _add(cls, torch, recs, pos, p, paired):
    n = recs.shape[0] // 2 if paired else recs.shape[0]
    d = _to_device(torch, recs, np.append(pos, np.uint32(0)), np.append(p, np.int32(0)))
    cls.add_device(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), n, paired)
    return d


@pytest.fixture(scope="module")
def small_ctx():
    torch = _torch()
    meta = json.load(open(os.path.join(GOLD, "golden.json")))
    prm = dict(meta["index"])
    for k in ("exons", "intron"):
        prm[k] = tuple(prm[k])
    ix = index.build_index(synth.transcriptome(synth.make_annotation(**prm)))
    ctx = api.Context(ix)
    yield torch, ix, ctx
    ctx.close()


@pytest.mark.parametrize("name", SETS)
def test_device_classes_golden(small_ctx, name):
    """Device class table over the golden records == the table the
    reference's own worker built from the same reads."""
    torch, ix, ctx = small_ctx
    c = np.load(os.path.join(GOLD, "candidates.npz"))
    d = np.load(os.path.join(GOLD, "classes.npz"))
    key = f"{name}_wb1"
    cls = api.Classes(ctx, max_classes=4096, max_list=1 << 16)
    try:
        _add(cls, torch, c[f"{key}_recs"], c[f"{key}_pos"], c[f"{key}_p"], name != "single")
        got = cls.fetch()
    finally:
        cls.close()
    want = oracle.ClassTable(d[f"{name}_ids"], d[f"{name}_counts"], d[f"{name}_ns"], d[f"{name}_ref_off"],
                             d[f"{name}_ref"], d[f"{name}_tx"], int(d[f"{name}_paired"][0]),
                             float(d[f"{name}_mean_frag"][0]))
    assert got.key() == want.key()


@pytest.fixture(scope="module")
def cfg1_ctx(config1):
    torch = _torch()
    ann, tx, ix = config1
    ctx = api.Context(ix)
    yield torch, ann, tx, ix, ctx
    ctx.close()


@pytest.mark.parametrize("wl", ["config1", "config4"])
@pytest.mark.parametrize("write_bam", [1, 0])
def test_classes_after_device_align(cfg1_ctx, oracle1, wl, write_bam):
    """Align on the device, classes from the device-resident results
    (add_last), batch by batch; equal to the oracle's add_class over its own
    records for the same reads, and to one table built in a single batch."""
    torch, ann, tx, ix, ctx = cfg1_ctx
    r1, r2 = workloads.pairs(wl, ann, tx, 30000, seed=211)
    want = oracle1.classes([oracle1.align_pairs(r1.copy(), r2.copy(), write_bam)])
    assert want.n_classes > 0
    cuts = (0, 5000, 17000, 30000)
    cls = api.Classes(ctx, max_classes=1 << 16, max_list=1 << 20)
    keep = []
    try:
        for a, b in zip(cuts[:-1], cuts[1:]):
            s1, s2 = r1.subset(np.arange(a, b)), r2.subset(np.arange(a, b))
            seq, off, lens = workloads.interleave(s1, s2)
            d = [torch.from_numpy(x).cuda() for x in (seq, off, lens)]
            keep.append(d)
            torch.cuda.synchronize()
            ctx.align_pairs_device(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), b - a,
                                   int(lens.max()), write_bam)
            cls.add_last(ctx)
        got = cls.fetch()
        t = cls.timing()
    finally:
        cls.close()
    assert got.key() == want.key()
    assert t["launches"] >= 4


def test_single_read_classes(cfg1_ctx, oracle1):
    """Single reads (align_single_read's merges before add_class)."""
    torch, ann, tx, ix, ctx = cfg1_ctx
    rs = synth.simulate_single(tx, 8000, seed=212)
    res = ctx.align_single(rs, 1)
    want = oracle1.classes([oracle1.align_single(rs.copy(), 1)], paired=False)
    cls = api.Classes(ctx, max_classes=4096, max_list=1 << 16)
    try:
        keep = _add(cls, torch, res.recs, res.pos_pool, res.p_pool, False)
        got = cls.fetch()
    finally:
        cls.close()
    del keep
    assert got.key() == want.key()


def test_class_table_capacity(cfg1_ctx, oracle1):
    """A table too small for the classes fails with ECAPACITY, not silently."""
    torch, ann, tx, ix, ctx = cfg1_ctx
    r1, r2 = workloads.pairs("config1", ann, tx, 8000, seed=213)
    res = ctx.align_pairs(r1, r2, 1)
    assert oracle1.classes([res]).n_classes > 2
    cls = api.Classes(ctx, max_classes=2, max_list=1 << 16)
    try:
        with pytest.raises(api.HeraGpuError) as e:
            keep = _add(cls, torch, res.recs, res.pos_pool, res.p_pool, True)
            del keep
        assert e.value.code == api.HERA_GPU_ECAPACITY
    finally:
        cls.close()


def test_classes_after_page_locked_fetch(cfg1_ctx, oracle1):
    """Fetching device-resident results into page-locked memory rebases the
    records on the device; fetching twice gives the same records, and the
    class table built afterwards from the same device records is unchanged."""
    import ctypes as C
    torch, ann, tx, ix, ctx = cfg1_ctx
    r1, r2 = workloads.pairs("config1", ann, tx, 20000, seed=214)
    want = oracle1.align_pairs(r1.copy(), r2.copy(), 1)
    seq, off, lens = workloads.interleave(r1, r2)
    d = [torch.from_numpy(x).cuda() for x in (seq, off, lens)]
    torch.cuda.synchronize()
    ctx.align_pairs_device(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), r1.n, int(lens.max()), 1)
    out = api.Result(2 * r1.n, 16 * r1.n + 1024, 16 * r1.n + 1024, 16 * r1.n + 1024)
    arrs = out.arrays()
    for a in arrs:
        api.host_register(a)
    try:
        for _ in range(2):
            ctx._check(ctx.lib.hera_gpu_fetch_result(ctx.h, C.byref(out.c)))
            assert out.canonical() == want.canonical()
    finally:
        for a in arrs:
            api.host_unregister(a)
    cls = api.Classes(ctx, max_classes=1 << 16, max_list=1 << 20)
    try:
        cls.add_last(ctx)
        got = cls.fetch()
    finally:
        cls.close()
    assert got.key() == oracle1.classes([want]).key()


def test_per_sample_classes_served_equal_alone(cfg1_ctx, oracle1):
    """Serving: one class table per sample, fed with the sample's served
    chunks in its own order (add_host), equals the table of the sample's
    chunks aligned alone, and the oracle's; the sample's EM abundances on
    the device are the oracle's (the reference's) bit for bit."""
    torch, ann, tx, ix, ctx = cfg1_ctx
    sizes = [3000, 11000, 700, 5000, 16000, 2500, 9000]
    models = ["config1", "config3", "config4"]
    chunks = []
    for k, n in enumerate(sizes):
        r1, r2 = workloads.pairs(models[k % 3], ann, tx, n, seed=300 + k)
        chunks.append((k % 3, r1, r2))
    alone = [ctx.align_pairs(r1, r2, 1) for _, r1, r2 in chunks]
    srv = api.Server(ctx, batch_pairs=4096, max_slots=3, write_bam=1, max_samples=4)
    try:
        tickets = [srv.submit(s, r1, r2) for s, r1, r2 in chunks]
        served = [srv.wait(t)[0] for t in tickets]
    finally:
        srv.close()
    for s in range(3):
        ks = [k for k, (si, _, _) in enumerate(chunks) if si == s]
        tabs, ems = [], []
        for src in (served, alone):
            cls = api.Classes(ctx, max_classes=1 << 14, max_list=1 << 18)
            try:
                for k in ks:
                    cls.add_result(src[k], paired=True)
                tabs.append(cls.fetch())
                ems.append(cls.em(ctx))
            finally:
                cls.close()
        want = oracle1.classes([oracle1.align_pairs(chunks[k][1].copy(), chunks[k][2].copy(), 1) for k in ks])
        assert tabs[0].key() == tabs[1].key() == want.key(), f"sample {s}"
        g0, o0, k0 = oracle1.em(want)
        for g, o, k, _ in ems:
            assert k == k0 and np.array_equal(_bits(g), _bits(g0)) and np.array_equal(_bits(o), _bits(o0))


def _bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.uint64)


@pytest.mark.parametrize("name", ["pairs100", "pairs_mixed", "pairs_n"])
def test_device_em_golden(small_ctx, name):
    """hera's EM on the device over the class table of the golden records:
    grama and overlap bit for bit as the reference's estimate_count left
    them on the same table."""
    torch, ix, ctx = small_ctx
    c = np.load(os.path.join(GOLD, "candidates.npz"))
    d = np.load(os.path.join(GOLD, "classes.npz"))
    key = f"{name}_wb1"
    cls = api.Classes(ctx, max_classes=4096, max_list=1 << 16)
    try:
        keep = _add(cls, torch, c[f"{key}_recs"], c[f"{key}_pos"], c[f"{key}_p"], True)
        g, o, rounds, ms = cls.em(ctx)
    finally:
        cls.close()
    del keep
    assert np.array_equal(_bits(g), _bits(d[f"{name}_em_grama"]))
    assert np.array_equal(_bits(o), _bits(d[f"{name}_em_overlap"]))
    assert rounds >= 50 and ms > 0


def test_device_em_after_align(cfg1_ctx, oracle1):
    """Align, classes and EM all on the device; equal to the oracle's EM
    (pinned to the reference's) over the oracle's own classes."""
    torch, ann, tx, ix, ctx = cfg1_ctx
    r1, r2 = workloads.pairs("config4", ann, tx, 20000, seed=215)
    want_t = oracle1.classes([oracle1.align_pairs(r1.copy(), r2.copy(), 1)])
    g0, o0, k0 = oracle1.em(want_t)
    seq, off, lens = workloads.interleave(r1, r2)
    dv = [torch.from_numpy(x).cuda() for x in (seq, off, lens)]
    torch.cuda.synchronize()
    ctx.align_pairs_device(dv[0].data_ptr(), dv[1].data_ptr(), dv[2].data_ptr(), r1.n, int(lens.max()), 1)
    cls = api.Classes(ctx, max_classes=1 << 16, max_list=1 << 20)
    try:
        cls.add_last(ctx)
        g, o, k, _ = cls.em(ctx)
    finally:
        cls.close()
    assert k == k0
    assert np.array_equal(_bits(g), _bits(g0)) and np.array_equal(_bits(o), _bits(o0))


def test_device_em_loaded_table_past_minimum(cfg1_ctx, oracle1):
    """A class table loaded from the host (hera's own CLASS), on which
    SQUAREM runs past 50 rounds: same rounds and arrays as the oracle."""
    from tests import em_cases
    torch, ann, tx, ix, ctx = cfg1_ctx
    t = em_cases.slow_table(ix.n_trans)
    g0, o0, k0 = oracle1.em(t)
    assert k0 > 50
    cls = api.Classes(ctx, max_classes=1 << 12, max_list=1 << 14)
    try:
        cls.load(t)
        assert cls.fetch().key()[1:] == t.key()[1:]
        g, o, k, _ = cls.em(ctx)
    finally:
        cls.close()
    assert k == k0
    assert np.array_equal(_bits(g), _bits(g0)) and np.array_equal(_bits(o), _bits(o0))
