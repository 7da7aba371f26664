"""GPU parity: the CUDA path (through the C ABI) against the oracle, record
for record -- hit lists, errors, CIGARs, miss chars and pair flags must be
identical (integer/byte work: the bar is bit-exact)."""
import ctypes as C

import numpy as np
import pytest

from hera_b200 import synth, workloads

pytestmark = pytest.mark.gpu


def _assert_same(g, o, what=""):
    cg, co = g.canonical(), o.canonical()
    assert len(cg) == len(co)
    bad = [i for i in range(len(cg)) if cg[i] != co[i]]
    assert not bad, (f"{what}: {len(bad)}/{len(cg)} records differ; first {bad[0]}:\n"
                     f" gpu    {cg[bad[0]]}\n oracle {co[bad[0]]}")


@pytest.mark.parametrize("write_bam", [1, 0])
def test_pairs_config1(config1, oracle1, gpu_ctx1, write_bam):
    ann, tx, _ = config1
    r1, r2 = workloads.pairs("config1", ann, tx, 30000, seed=7)
    _assert_same(gpu_ctx1.align_pairs(r1, r2, write_bam),
                 oracle1.align_pairs(r1.copy(), r2.copy(), write_bam), "config1")


@pytest.mark.parametrize("write_bam", [1, 0])
def test_pairs_high_divergence(config1, oracle1, gpu_ctx1, write_bam):
    """2x150 bp, 3% substitutions, 1-8 bp indels, mutated loci: many mate
    rescues (ssw_align) and early-stopping gap DPs."""
    ann, tx, _ = config1
    r1, r2 = workloads.pairs("config4", ann, tx, 8000, seed=8)
    _assert_same(gpu_ctx1.align_pairs(r1, r2, write_bam),
                 oracle1.align_pairs(r1.copy(), r2.copy(), write_bam), "config4")


@pytest.mark.parametrize("write_bam", [1, 0])
def test_pairs_mixed_lengths(config1, oracle1, gpu_ctx1, write_bam):
    ann, tx, _ = config1
    r1, r2 = workloads.pairs("config3", ann, tx, 8000, seed=9)
    _assert_same(gpu_ctx1.align_pairs(r1, r2, write_bam),
                 oracle1.align_pairs(r1.copy(), r2.copy(), write_bam), "config3 pairs")


@pytest.mark.parametrize("write_bam", [1, 0])
def test_single_mixed_lengths(config1, oracle1, gpu_ctx1, write_bam):
    _, tx, _ = config1
    rs = workloads.singles("config3", tx, 10000, seed=10)
    _assert_same(gpu_ctx1.align_single(rs, write_bam), oracle1.align_single(rs.copy(), write_bam),
                 "config3 single")


def test_pairs_with_n(config1, oracle1, gpu_ctx1):
    """N bytes bleed into the neighbouring k-mer bits and match each other in
    both DPs."""
    _, tx, _ = config1
    r1, r2 = synth.simulate_pairs(tx, 6000, seed=15, read_len=100, sub_rate=0.01)
    rng = np.random.default_rng(3)
    for rs in (r1, r2):
        rs.seq[rng.random(rs.seq.shape[0]) < 0.01] = ord("N")
    for wb in (1, 0):
        _assert_same(gpu_ctx1.align_pairs(r1, r2, wb), oracle1.align_pairs(r1.copy(), r2.copy(), wb),
                     f"N reads wb={wb}")


def test_pairs_lowercase(config1, oracle1, gpu_ctx1):
    _, tx, _ = config1
    r1, r2 = synth.simulate_pairs(tx, 3000, seed=16, read_len=100, sub_rate=0.01)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    r1.seq[:] = np.where(np.isin(r1.seq, acgt), r1.seq + 32, r1.seq)
    _assert_same(gpu_ctx1.align_pairs(r1, r2, 0), oracle1.align_pairs(r1.copy(), r2.copy(), 0), "lower")


def test_pairs_long_reads(config1, oracle1, gpu_ctx1):
    """Reads > 252 bp: the rescue DP's u8 cells saturate exactly as hera's
    SSE2 lanes do (no 16-bit rerun)."""
    _, tx, _ = config1
    r1, r2 = synth.simulate_pairs(tx, 1500, seed=17, read_len=260, frag_mu=400, frag_sd=30,
                                  sub_rate=0.02, indel_rate=0.002)
    for wb in (1, 0):
        _assert_same(gpu_ctx1.align_pairs(r1, r2, wb), oracle1.align_pairs(r1.copy(), r2.copy(), wb),
                     f"260 bp wb={wb}")


def test_batch_split_invariance(config1, gpu_ctx1):
    """Results do not depend on how pairs are split into device passes."""
    from hera_b200 import api
    ann, tx, ix = config1
    r1, r2 = workloads.pairs("config1", ann, tx, 5000, seed=21)
    a = gpu_ctx1.align_pairs(r1, r2, 0).canonical()
    small = api.Context(ix, max_batch=777, path=gpu_ctx1.path)
    try:
        b = small.align_pairs(r1, r2, 0).canonical()
    finally:
        small.close()
    assert a == b


def test_device_resident_entry(config1, gpu_ctx1):
    import torch
    ann, tx, _ = config1
    r1, r2 = workloads.pairs("config1", ann, tx, 4000, seed=22)
    flat = gpu_ctx1.align_pairs(r1, r2, 1).canonical()
    seq, off, lens = workloads.interleave(r1, r2)
    d = [torch.from_numpy(x).cuda() for x in (seq, off, lens)]
    torch.cuda.synchronize()
    gpu_ctx1.align_pairs_device(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), r1.n,
                                int(lens.max()), 1, None)
    dev = gpu_ctx1.fetch(2 * r1.n).canonical()
    assert dev == flat


class ReadInf(C.Structure):
    _fields_ = [("seq", C.c_char_p), ("name", C.c_char_p), ("qual", C.c_char_p), ("len", C.c_int32)]


class Cigar(C.Structure):
    _fields_ = [("n_cigar", C.c_ushort), ("n_miss", C.c_ushort), ("count", C.POINTER(C.c_ushort)),
                ("type", C.POINTER(C.c_char)), ("miss", C.POINTER(C.c_char))]


class Candidate(C.Structure):
    _fields_ = [("p", C.POINTER(C.c_int) * 2), ("pos", C.POINTER(C.c_uint) * 2), ("n", C.c_uint * 2),
                ("err", C.c_int * 2), ("cigar", C.POINTER(Cigar) * 2), ("pair", C.c_int)]


def test_dropin_candidate_entry(config1, oracle1, gpu_ctx1):
    """hera_gpu_align_pairs returns hera's own Candidate structs (malloc'd,
    reference layout) equal to the flat records; lower-case reads come back
    upper-case like the reference leaves them."""
    ann, tx, _ = config1
    r1, r2 = workloads.pairs("config1", ann, tx, 1500, seed=23)
    r1.seq[:50] = np.where(r1.seq[:50] == ord("A"), ord("a"), r1.seq[:50])
    o = oracle1.align_pairs(r1.copy(), r2.copy(), 0).canonical()
    n = r1.n
    bufs = []
    arr1, arr2 = (ReadInf * n)(), (ReadInf * n)()
    for rs, arr in ((r1, arr1), (r2, arr2)):
        for i in range(n):
            b = C.create_string_buffer(rs.read(i))
            bufs.append(b)
            arr[i].seq = C.cast(b, C.c_char_p)
            arr[i].len = int(rs.len[i])
    out = (C.POINTER(Candidate) * (2 * n))()
    lib = gpu_ctx1.lib
    lib.hera_gpu_align_pairs.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int, C.c_void_p]
    rc = lib.hera_gpu_align_pairs(gpu_ctx1.h, arr1, arr2, n, 0, out)
    assert rc == 0
    chars = "MIDNSHP=XB"
    for i in range(2 * n):
        c = out[i].contents
        strands = []
        for s in range(2):
            k = c.n[s]
            g = c.cigar[s].contents
            cig = "".join(f"{g.count[j]}{chars[g.type[j][0]]}" for j in range(g.n_cigar))
            miss = bytes(g.miss[j][0] for j in range(g.n_miss))
            strands.append((k, c.err[s], tuple(c.pos[s][j] for j in range(k)),
                            tuple(c.p[s][j] for j in range(k)), cig, miss))
        assert (c.pair, tuple(strands)) == o[i], i
    assert bufs[0].value.upper() == bufs[0].value


def _candidates(lib, h, r1, r2, write_bam):
    """hera_gpu_align_pairs on (r1, r2) as read_inf arrays; the Candidates
    decoded into the oracle's canonical tuples, then freed."""
    n = r1.n
    bufs = []
    arr1, arr2 = (ReadInf * n)(), (ReadInf * n)()
    for rs, arr in ((r1, arr1), (r2, arr2)):
        for i in range(n):
            b = C.create_string_buffer(rs.read(i))
            bufs.append(b)
            arr[i].seq = C.cast(b, C.c_char_p)
            arr[i].len = int(rs.len[i])
    out = (C.POINTER(Candidate) * (2 * n))()
    rc = lib.hera_gpu_align_pairs(h, arr1, arr2, n, write_bam, out)
    assert rc == 0
    chars = "MIDNSHP=XB"
    got = []
    for i in range(2 * n):
        c = out[i].contents
        strands = []
        for s in range(2):
            k = c.n[s]
            g = c.cigar[s].contents
            cig = "".join(f"{g.count[j]}{chars[g.type[j][0]]}" for j in range(g.n_cigar))
            miss = bytes(g.miss[j][0] for j in range(g.n_miss))
            strands.append((k, c.err[s], tuple(c.pos[s][j] for j in range(k)),
                            tuple(c.p[s][j] for j in range(k)), cig, miss))
        got.append((c.pair, tuple(strands)))
    lib.hera_gpu_free_candidates(out, 2 * n)
    return got


@pytest.mark.parametrize("write_bam", [1, 0])
def test_dropin_calls_from_threads_combine(config1, oracle1, gpu_ctx1, write_bam):
    """hera's -t N workers call hera_gpu_align_pairs on one context at the
    same time: the calls are combined into shared device batches and every
    call still gets exactly its own pairs' Candidates."""
    import threading
    ann, tx, _ = config1
    r1, r2 = workloads.pairs("config1", ann, tx, 4800, seed=29)
    lib = gpu_ctx1.lib
    lib.hera_gpu_align_pairs.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int, C.c_void_p]
    lib.hera_gpu_free_candidates.argtypes = [C.c_void_p, C.c_int64]
    want = oracle1.align_pairs(r1.copy(), r2.copy(), write_bam).canonical()
    parts = np.array_split(np.arange(r1.n), 12)
    got, errs = [None] * len(parts), []

    def work(k):
        try:
            idx = parts[k]
            got[k] = _candidates(lib, gpu_ctx1.h, r1.subset(idx), r2.subset(idx), write_bam)
        except Exception as e:   # reported below
            errs.append(e)
    for _ in range(3):
        th = [threading.Thread(target=work, args=(k,)) for k in range(len(parts))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert not errs, errs[0]
        for k, idx in enumerate(parts):
            assert got[k] == [want[j] for i in idx for j in (2 * i, 2 * i + 1)], k


@pytest.mark.parametrize("shape", [(1, 1), (16, 8), (3, 2)])
def test_launch_shapes_do_not_change_results(config1, oracle1, shape):
    """The autotuner's choices (build residency, rescue calls per block) only
    change speed: pinned extreme shapes give the oracle's records."""
    if not __import__("torch").cuda.is_available():
        pytest.skip("no CUDA device")
    from hera_b200 import api
    ann, tx, ix = config1
    ctx = api.Context(ix, max_batch=1 << 16)
    try:
        ctx.set_tuning(*shape)
        r1, r2 = workloads.pairs("config4", ann, tx, 6000, seed=31)
        _assert_same(ctx.align_pairs(r1, r2, 0), oracle1.align_pairs(r1.copy(), r2.copy(), 0),
                     f"shape {shape}")
        t = ctx.tuning()
        assert t["state"] == "pinned"
        assert (t["build_blocks_per_sm"], t["rescue_warps_per_block"]) == shape
    finally:
        ctx.close()


def test_autotuner_picks_a_timed_candidate(config1, oracle1):
    """A batch of at least 16384 pairs on one lane makes the context time
    every build-residency candidate and keep the fastest; results stay the
    oracle's."""
    if not __import__("torch").cuda.is_available():
        pytest.skip("no CUDA device")
    from hera_b200 import api
    ann, tx, ix = config1
    ctx = api.Context(ix, max_batch=1 << 16, lanes=1)
    try:
        assert ctx.tuning()["state"] == "defaults"
        r1, r2 = workloads.pairs("config1", ann, tx, 20000, seed=32)
        _assert_same(ctx.align_pairs(r1, r2, 1), oracle1.align_pairs(r1.copy(), r2.copy(), 1), "tuned")
        t = ctx.tuning()
        assert t["state"] == "autotuned"
        trials = t["build_trials_ms"]
        assert len(trials) >= 4 and all(v > 0 for v in trials.values())
        assert t["build_blocks_per_sm"] == min(trials, key=trials.get)
    finally:
        ctx.close()


def test_page_locked_buffers_same_records(config1, gpu_ctx1):
    """Page-locked reads and result pools take the direct copy paths (no
    pinned staging; records rebased on the device) and give the same
    records as pageable ones."""
    from hera_b200 import api
    ann, tx, _ = config1
    r1, r2 = workloads.pairs("config4", ann, tx, 12000, seed=41)
    ref = gpu_ctx1.align_pairs(r1, r2, 0)
    out = gpu_ctx1.align_pairs(r1, r2, 0)
    arrs = [r1.seq, r2.seq] + out.arrays()
    for a in arrs:
        api.host_register(a)
    try:
        res = gpu_ctx1.align_pairs(r1, r2, 0, out=out)
        assert res.canonical() == ref.canonical()
        res = gpu_ctx1.align_pairs(r1, r2, 0, out=out)   # a second call over the same buffers
        assert res.canonical() == ref.canonical()
    finally:
        for a in arrs:
            api.host_unregister(a)


@pytest.fixture(scope="module", params=["batched", "plain"])
def ctx2s(request, config2s):
    from hera_b200 import api
    ctx = api.Context(config2s[2], path=request.param)
    yield ctx
    ctx.close()


@pytest.fixture(scope="module")
def oracle2s(config2s):
    import oracle
    return oracle.Oracle(config2s[2])


@pytest.mark.parametrize("write_bam", [1, 0])
def test_pairs_config2s(config2s, oracle2s, ctx2s, write_bam):
    """Config 2's isoform structure (20k transcripts: buckets with several
    entries, long occurrence lists, many-isoform merge_sort ties), 60k pairs
    of its read model, record for record."""
    ann, tx, _ = config2s
    r1, r2 = workloads.pairs("config2s", ann, tx, 60000, seed=17)
    _assert_same(ctx2s.align_pairs(r1, r2, write_bam), oracle2s.align_pairs(r1.copy(), r2.copy(), write_bam),
                 f"config2s wb={write_bam}")


@pytest.fixture(scope="module", params=["batched", "plain"])
def ctx_family(request, family):
    from hera_b200 import api
    ctx = api.Context(family[1], path=request.param)
    yield ctx
    ctx.close()


@pytest.mark.parametrize("mate2_random", [False, True])
def test_pairs_past_list_capacities(family, ctx_family, mate2_random):
    """Reads with 96 hits a strand and over 256 anchors at seed spacing 14,
    among ordinary reads, and mates rescued over every family member: the
    pairs past the first pass's per-read capacities run a second, wide pass
    and every record equals the oracle's (no capacity error)."""
    import oracle
    tx, ix = family
    orc = oracle.Oracle(ix)
    f1, f2 = synth.family_pairs(tx, 500, seed=18, shared=600, mate2_random=mate2_random)
    o1, o2 = synth.simulate_pairs(tx, 1500, seed=19, read_len=100, sub_rate=0.01)
    r1, r2 = synth.concat_pairs([(f1, f2), (o1, o2)], seed=20)
    for wb in (1, 0):
        got = ctx_family.align_pairs(r1, r2, wb)
        want = orc.align_pairs(r1.copy(), r2.copy(), wb)
        assert int(want.recs["n"].max()) > 64
        _assert_same(got, want, f"family mate2_random={mate2_random} wb={wb}")


def test_single_past_list_capacities(family, ctx_family):
    import oracle
    tx, ix = family
    orc = oracle.Oracle(ix)
    f1, _ = synth.family_pairs(tx, 400, seed=21, shared=600)
    for wb in (1, 0):
        _assert_same(ctx_family.align_single(f1, wb), orc.align_single(f1.copy(), wb), f"family single wb={wb}")


def test_async_calls_equal_sync(config1, oracle1):
    """Two asynchronous flat calls in flight at once (each on its own lane
    group) give the records of the synchronous call; a third submit is
    refused while both are in flight."""
    if not __import__("torch").cuda.is_available():
        pytest.skip("no CUDA device")
    from hera_b200 import api
    ann, tx, ix = config1
    ctx = api.Context(ix, max_batch=1 << 14, lanes=2)
    try:
        sets = [workloads.pairs(wl, ann, tx, 9000, seed=70 + k) for k, wl in enumerate(("config1", "config4", "config3"))]
        want = [ctx.align_pairs(r1, r2, 0).canonical() for r1, r2 in sets]
        outs = [api.Result(2 * 9000, 1 << 20, 1 << 20, 1 << 20) for _ in range(2)]
        t0 = ctx.submit_pairs(*sets[0], 0, outs[0])
        t1 = ctx.submit_pairs(*sets[1], 0, outs[1])
        with pytest.raises(api.HeraGpuError):
            ctx.submit_pairs(*sets[2], 0, api.Result(2 * 9000, 1 << 20, 1 << 20, 1 << 20))
        assert ctx.complete_pairs(t0).canonical() == want[0]
        t2 = ctx.submit_pairs(*sets[2], 0, outs[0])
        assert ctx.complete_pairs(t1).canonical() == want[1]
        assert ctx.complete_pairs(t2).canonical() == want[2]
        assert want[1] == oracle1.align_pairs(sets[1][0].copy(), sets[1][1].copy(), 0).canonical()
    finally:
        ctx.close()
