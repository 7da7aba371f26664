"""The allocation-free entry point (hera_gpu_align_pairs_device_noalloc).

Some callers of this library cannot allocate device memory while they
align: they run inside a memory pool they do not own, or under a hard memory
budget where a cudaMalloc would fail or synchronise the device.  For them
the library has one entry point that allocates nothing: it runs the same
kernels as hera_gpu_align_pairs_device with all of its working memory --
DP jobs, per-pair state, queues and mate-rescue outputs -- in one static
device array (limit: 1024 pairs per call), and writes its records into
device buffers the caller owns.  This file checks, through the C ABI, that
its records are identical to those of hera_gpu_align_pairs_device on two
calls in a row (the array keeps the previous call's contents), that
oversized batches are refused, and that a batch whose working set outgrows
the static array fails cleanly (no pool sizes claimed) and leaves the next
call correct.  It is collected last so that a run stopping at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from hera_b200 import api, workloads

pytestmark = pytest.mark.gpu

MAX_PAIRS = 1024


def _device_out(torch, n, cap):
    recs = torch.empty(2 * n * api.REC_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    pos = torch.empty(cap, dtype=torch.int32, device="cuda")
    p = torch.empty(cap, dtype=torch.int32, device="cuda")
    ops = torch.empty(cap, dtype=torch.int32, device="cuda")
    miss = torch.empty(cap, dtype=torch.uint8, device="cuda")
    res = api._Result(recs.data_ptr(), pos.data_ptr(), p.data_ptr(), ops.data_ptr(), miss.data_ptr(),
                      cap, cap, cap, 0, 0, 0)
    return res, (recs, pos, p, ops, miss)


def _to_host(res, bufs, n):
    recs, pos, p, ops, miss = bufs
    out = api.Result(2 * n, 1, 1, 1)
    out.recs[:] = np.frombuffer(recs.cpu().numpy().tobytes(), dtype=api.REC_DTYPE)
    out.pos_pool = pos.cpu().numpy().view(np.uint32)
    out.p_pool = p.cpu().numpy()
    out.op_pool = ops.cpu().numpy().view(np.uint32)
    out.miss_pool = miss.cpu().numpy()
    return out.canonical()


@pytest.fixture(scope="module")
def setup():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ann, tx, ix = workloads.build("config1")
    ctx = api.Context(ix)
    lib = ctx.lib
    lib.hera_gpu_align_pairs_device_noalloc.restype = C.c_int
    lib.hera_gpu_align_pairs_device_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                       C.c_int32, C.c_int32, C.c_int, C.POINTER(api._Result),
                                                       C.c_void_p]
    yield torch, ann, tx, ctx
    ctx.close()


def _device_reads(torch, r1, r2):
    seq, off, lens = workloads.interleave(r1, r2)
    d = [torch.from_numpy(x).cuda() for x in (seq, off, lens)]
    torch.cuda.synchronize()
    return d, int(lens.max())


@pytest.mark.parametrize("write_bam", [1, 0])
def test_noalloc_matches_device_entry_twice(setup, write_bam):
    torch, ann, tx, ctx = setup
    # two different batches in a row: the second call must not depend on
    # what the first left in the shared static array
    for seed, wl in ((41, "config4"), (42, "config1")):
        r1, r2 = workloads.pairs(wl, ann, tx, MAX_PAIRS, seed=seed)
        (s, o, ln), max_len = _device_reads(torch, r1, r2)
        ctx.align_pairs_device(s.data_ptr(), o.data_ptr(), ln.data_ptr(), r1.n, max_len, write_bam, None)
        want = ctx.fetch(2 * r1.n).canonical()
        res, bufs = _device_out(torch, r1.n, 64 * r1.n)
        rc = ctx.lib.hera_gpu_align_pairs_device_noalloc(ctx.h, s.data_ptr(), o.data_ptr(), ln.data_ptr(),
                                                          r1.n, max_len, write_bam, C.byref(res), None)
        assert rc == 0, ctx.lib.hera_gpu_last_error(ctx.h).decode()
        torch.cuda.synchronize()
        got = _to_host(res, bufs, r1.n)
        assert len(got) == len(want) == 2 * r1.n
        bad = [i for i in range(len(want)) if got[i] != want[i]]
        assert not bad, f"{wl}: {len(bad)} records differ, first {bad[0]}: {got[bad[0]]} vs {want[bad[0]]}"


def test_noalloc_rejects_oversized_batch(setup):
    torch, ann, tx, ctx = setup
    r1, r2 = workloads.pairs("config1", ann, tx, MAX_PAIRS + 1, seed=43)
    (s, o, ln), max_len = _device_reads(torch, r1, r2)
    res, bufs = _device_out(torch, r1.n, 16)
    rc = ctx.lib.hera_gpu_align_pairs_device_noalloc(ctx.h, s.data_ptr(), o.data_ptr(), ln.data_ptr(),
                                                      r1.n, max_len, 1, C.byref(res), None)
    assert rc == -4
    assert b"1024" in ctx.lib.hera_gpu_last_error(ctx.h)


def test_noalloc_reports_small_output(setup):
    torch, ann, tx, ctx = setup
    r1, r2 = workloads.pairs("config1", ann, tx, 200, seed=44)
    (s, o, ln), max_len = _device_reads(torch, r1, r2)
    res, bufs = _device_out(torch, r1.n, 4)
    rc = ctx.lib.hera_gpu_align_pairs_device_noalloc(ctx.h, s.data_ptr(), o.data_ptr(), ln.data_ptr(),
                                                      r1.n, max_len, 1, C.byref(res), None)
    assert rc == -5
    assert res.list_used > 4


def test_noalloc_scratch_overflow_then_normal_call(setup):
    """1024 pairs from a sequence shared by 48 transcripts: every
    get_position call forms 48 chains, far more than the static array holds
    for 1024 pairs.  The call fails with HERA_GPU_ECAPACITY, says to align
    fewer pairs, and claims no pool sizes; the next call, on ordinary
    reads, still equals hera_gpu_align_pairs_device."""
    torch, ann, tx, ctx = setup
    from hera_b200 import index, synth
    ftx = synth.family_transcriptome(5, families=((48, 600),), n_other=20)
    fctx = api.Context(index.build_index(ftx))
    try:
        lib = fctx.lib
        f1, f2 = synth.family_pairs(ftx, MAX_PAIRS, seed=6, shared=600)
        (s, o, ln), max_len = _device_reads(torch, f1, f2)
        res, bufs = _device_out(torch, f1.n, 64 * f1.n)
        rc = lib.hera_gpu_align_pairs_device_noalloc(fctx.h, s.data_ptr(), o.data_ptr(), ln.data_ptr(),
                                                     f1.n, max_len, 1, C.byref(res), None)
        msg = lib.hera_gpu_last_error(fctx.h).decode()
        assert rc == -5, msg
        assert "fewer pairs" in msg, msg
        assert res.list_used == res.op_used == res.miss_used == 0
        # the same context, ordinary reads from its own transcripts
        r1, r2 = synth.simulate_pairs(ftx, 300, seed=7, read_len=100, sub_rate=0.005)
        (s, o, ln), max_len = _device_reads(torch, r1, r2)
        fctx.align_pairs_device(s.data_ptr(), o.data_ptr(), ln.data_ptr(), r1.n, max_len, 1, None)
        want = fctx.fetch(2 * r1.n).canonical()
        res, bufs = _device_out(torch, r1.n, 256 * r1.n)
        rc = lib.hera_gpu_align_pairs_device_noalloc(fctx.h, s.data_ptr(), o.data_ptr(), ln.data_ptr(),
                                                     r1.n, max_len, 1, C.byref(res), None)
        assert rc == 0, lib.hera_gpu_last_error(fctx.h).decode()
        torch.cuda.synchronize()
        assert _to_host(res, bufs, r1.n) == want
    finally:
        fctx.close()


def test_noalloc_output_pools_exact_capacity(setup):
    """Pools given exactly the sizes a batch needs are enough (nothing is
    written at or past the capacity); one entry less is refused with the
    sizes needed."""
    torch, ann, tx, ctx = setup
    r1, r2 = workloads.pairs("config1", ann, tx, 300, seed=45)
    (s, o, ln), max_len = _device_reads(torch, r1, r2)
    res, bufs = _device_out(torch, r1.n, 64 * r1.n)
    rc = ctx.lib.hera_gpu_align_pairs_device_noalloc(ctx.h, s.data_ptr(), o.data_ptr(), ln.data_ptr(),
                                                      r1.n, max_len, 0, C.byref(res), None)
    assert rc == 0
    torch.cuda.synchronize()
    want = _to_host(res, bufs, r1.n)
    need = (res.list_used, res.op_used, res.miss_used)
    assert min(need) > 0
    res2, bufs2 = _device_out(torch, r1.n, max(need))
    res2.list_cap, res2.op_cap, res2.miss_cap = need
    rc = ctx.lib.hera_gpu_align_pairs_device_noalloc(ctx.h, s.data_ptr(), o.data_ptr(), ln.data_ptr(),
                                                      r1.n, max_len, 0, C.byref(res2), None)
    assert rc == 0, ctx.lib.hera_gpu_last_error(ctx.h).decode()
    torch.cuda.synchronize()
    assert _to_host(res2, bufs2, r1.n) == want
    res3, bufs3 = _device_out(torch, r1.n, max(need))
    res3.list_cap, res3.op_cap, res3.miss_cap = need[0] - 1, need[1], need[2]
    rc = ctx.lib.hera_gpu_align_pairs_device_noalloc(ctx.h, s.data_ptr(), o.data_ptr(), ln.data_ptr(),
                                                      r1.n, max_len, 0, C.byref(res3), None)
    assert rc == -5
    assert (res3.list_used, res3.op_used, res3.miss_used) == need
