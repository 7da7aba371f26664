"""FASTQ chunk parsing (hera's get_read_from_fq_buffer, src/read.c:11-63, in
the read loops of align_pool_pair / align_pool_single,
src/hash_align.c:1878-1929, 1966-1998).

CPU: the oracle's restatement against the golden vectors made by the
reference's own reader, against the reference live where it was built here,
and the reader's side effects (hera_gpu_fastq_read_inf, host code).
GPU: the device parse against the same golden vectors and the oracle, on
malformed chunks, on chunks spanning many 8 KiB tiles, and parse + align
against hera_gpu_align_pairs_flat on the same reads."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from hera_b200 import api, build, synth, workloads

from . import fastq_cases

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fastq.npz")


def _golden_pairs():
    z = np.load(GOLDEN)
    lo, ro, so = z["pair_left_off"], z["pair_right_off"], z["pair_recs_off"]
    for k in range(len(lo) - 1):
        left = z["pair_left"][lo[k]:lo[k + 1]].tobytes()
        right = z["pair_right"][ro[k]:ro[k + 1]].tobytes()
        yield left, right, tuple(int(x) for x in z["pair_result"][k]), z["pair_recs"][so[k]:so[k + 1]]


def _golden_singles():
    z = np.load(GOLDEN)
    bo, so = z["single_off"], z["single_recs_off"]
    for k in range(len(bo) - 1):
        yield (z["single_buf"][bo[k]:bo[k + 1]].tobytes(), tuple(int(x) for x in z["single_result"][k]),
               z["single_recs"][so[k]:so[k + 1]])


def _same(a, b) -> bool:
    return a[0] == b[0] and a[2:] == b[2:] and np.array_equal(a[1], b[1])


# ---- CPU ---------------------------------------------------------------------

def test_oracle_matches_golden():
    n = 0
    for left, right, (st, npairs, bf, br), recs in _golden_pairs():
        got = oracle.parse_fq_pairs(left, right)
        assert (got[0], got[2], got[3], got[4]) == (st, npairs, bf, br)
        assert np.array_equal(got[1], recs)
        n += 1
    for buf, (st, nreads, _, br), recs in _golden_singles():
        got = oracle.parse_fq_single(buf)
        assert (got[0], got[2], got[4]) == (st, nreads, br)
        assert np.array_equal(got[1], recs)
        n += 1
    assert n > 200


@pytest.mark.skipif(not oracle.reference_available(), reason="reference not built")
def test_oracle_matches_reference_live():
    for left, right in fastq_cases.pair_cases(31, 300):
        assert _same(oracle.parse_fq_pairs(left, right), oracle.ref_parse_fq_pairs(left, right))
    for buf in fastq_cases.single_cases(32, 150):
        assert _same(oracle.parse_fq_single(buf), oracle.ref_parse_fq_single(buf))


@pytest.mark.skipif(not oracle.reference_available() or not os.path.exists(build.LIB),
                    reason="reference or library not built")
def test_read_inf_side_effects_match_reference():
    """hera_gpu_fastq_read_inf leaves the buffers as the reader does and
    points each read_inf at the reader's strings (host code, no GPU)."""
    lib = api.load_library()
    lib.hera_gpu_fastq_read_inf.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int32, C.c_int32,
                                            C.c_void_p]

    class ReadInf(C.Structure):
        _fields_ = [("seq", C.c_void_p), ("name", C.c_void_p), ("qual", C.c_void_p), ("len", C.c_int32)]

    checked = 0
    for left, right in fastq_cases.pair_cases(33, 120):
        bufs = []
        rc, recs, n, _, _ = oracle.ref_parse_fq_pairs(left, right, buffers=bufs)
        if rc != 0:
            continue
        for side, raw in ((0, left), (1, right)):
            a = np.frombuffer(raw, np.uint8).copy()
            out = (ReadInf * max(n, 1))()
            assert lib.hera_gpu_fastq_read_inf(a.ctypes.data, a.size, recs[side:].ctypes.data, n, 2, out) == 0
            # the reader writes its NULs only up to where it stopped; past the
            # last read both buffers are untouched
            assert a.tobytes() == bufs[side]
            base = a.ctypes.data
            for i in range(n):
                r = recs[2 * i + side]
                assert out[i].seq - base == r["seq"] and out[i].name - base == r["name"]
                assert out[i].qual - base == r["qual"] and out[i].len == r["len"]
        checked += 1
    assert checked > 40


# ---- GPU ---------------------------------------------------------------------

def _device_pairs(ctx, left, right):
    try:
        recs = ctx.parse_fastq_pairs(left, right)
        return 0, recs, recs.shape[0] // 2, 0, -1
    except api.FastqFormatError as e:
        return -1, np.zeros(0, api.FQ_DTYPE), 0, e.bad_file, e.bad_read


def _device_single(ctx, buf):
    try:
        recs = ctx.parse_fastq_single(buf)
        return 0, recs, recs.shape[0], 0, -1
    except api.FastqFormatError as e:
        return -1, np.zeros(0, api.FQ_DTYPE), 0, 0, e.bad_read


@pytest.fixture(scope="module")
def fq_ctx(config1):
    if not __import__("torch").cuda.is_available():
        pytest.skip("no CUDA device")
    ctx = api.Context(config1[2])
    yield ctx
    ctx.close()


@pytest.mark.gpu
def test_device_parse_golden(fq_ctx):
    for left, right, (st, npairs, bf, br), recs in _golden_pairs():
        got = _device_pairs(fq_ctx, left, right)
        assert (got[0], got[2], got[3], got[4]) == (st, npairs, bf, br)
        assert np.array_equal(got[1], recs)
    for buf, (st, nreads, _, br), recs in _golden_singles():
        got = _device_single(fq_ctx, buf)
        assert (got[0], got[2], got[4]) == (st, nreads, br)
        assert np.array_equal(got[1], recs)


@pytest.mark.gpu
def test_device_parse_fuzz_matches_oracle(fq_ctx):
    for left, right in fastq_cases.pair_cases(34, 250):
        assert _same(_device_pairs(fq_ctx, left, right), oracle.parse_fq_pairs(left, right))
    for buf in fastq_cases.single_cases(35, 120):
        assert _same(_device_single(fq_ctx, buf), oracle.parse_fq_single(buf))


@pytest.mark.gpu
def test_device_parse_large_chunks(fq_ctx, config1):
    """Chunks of many tiles (reads of 50-150 bp), whole, cut short, with a
    blank line after, a NUL inside, and a read spoiled far from the start."""
    ann, tx, _ = config1
    r1, r2 = workloads.pairs("config3", ann, tx, 60000, seed=41)
    left, right = synth.fastq_bytes(r1, 1), synth.fastq_bytes(r2, 2)
    assert len(left) > 64 * 8192
    cases = [(left, right), (left, right[:len(right) - 1]), (left[:len(left) // 2 + 7], right),
             (left + b"\n", right), (left[:300001] + b"\0" + left[300002:], right),
             (left, right[:777777] + b"X" + right[777778:])]
    for l, r in cases:
        assert _same(_device_pairs(fq_ctx, l, r), oracle.parse_fq_pairs(l, r, cap=70000))
    rs = workloads.singles("config3", tx, 50000, seed=42)
    s = synth.fastq_bytes(rs)
    assert _same(_device_single(fq_ctx, s), oracle.parse_fq_single(s, cap=60000))
    st = fq_ctx.fastq_stats()
    assert st["bytes"] == len(s) and st["reads"] == 50000 and st["parse_ms"] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("wl", ["config1", "config4"])
def test_align_fastq_equals_align_pairs(fq_ctx, config1, wl):
    ann, tx, _ = config1
    r1, r2 = workloads.pairs(wl, ann, tx, 6000, seed=43)
    left, right = synth.fastq_bytes(r1, 1), synth.fastq_bytes(r2, 2)
    for wb in (1, 0):
        res, recs = fq_ctx.align_fastq_pairs(left, right, wb)
        assert recs.shape[0] == 2 * r1.n
        assert np.array_equal(recs, oracle.parse_fq_pairs(left, right, cap=7000)[1])
        want = fq_ctx.align_pairs(r1, r2, wb)
        assert res.canonical() == want.canonical()
    # the reads of a parse, over the chunk buffers, through the host API
    recs = fq_ctx.parse_fastq_pairs(left, right)
    a, b = api.FastqReads(left, recs[0::2]), api.FastqReads(right, recs[1::2])
    assert fq_ctx.align_pairs(a, b, 1).canonical() == fq_ctx.align_pairs(r1, r2, 1).canonical()


@pytest.mark.gpu
def test_align_fastq_rejects_like_reference(fq_ctx, config1):
    ann, tx, _ = config1
    r1, r2 = workloads.pairs("config1", ann, tx, 500, seed=44)
    left, right = synth.fastq_bytes(r1, 1), synth.fastq_bytes(r2, 2)
    k = -1
    for _ in range(3):   # the third read's '+' line of file 2
        k = right.index(b"\n+\n", k + 1)
    bad = right[:k + 1] + b"-" + right[k + 2:]
    want = oracle.parse_fq_pairs(left, bad)
    assert want[0] == -1 and want[3:] == (2, 2)
    with pytest.raises(api.FastqFormatError) as e:
        fq_ctx.align_fastq_pairs(left, bad, 1)
    assert (e.value.bad_file, e.value.bad_read) == (2, 2)


@pytest.mark.gpu
def test_parse_grows_record_array(fq_ctx):
    """Many one-base reads: more reads than the first record array holds,
    so the call reports the count and is repeated with room for all."""
    n = 12000
    left = b"".join(b"@%d\nA\n+\nI\n" % i for i in range(n))
    right = b"".join(b"@%d\nC\n+\nI\n" % i for i in range(n))
    recs = fq_ctx.parse_fastq_pairs(left, right)
    assert recs.shape[0] == 2 * n
    assert np.array_equal(recs, oracle.parse_fq_pairs(left, right)[1])


@pytest.mark.gpu
def test_align_fastq_rejects_overlong_read(fq_ctx):
    """Reads the aligner cannot take (longer than HERA_GPU_MAX_READ) are
    refused with HERA_GPU_EINVAL, after a parse that accepts them."""
    long = b"A" * (api.MAX_READ + 1)
    left = b"@a\n" + long + b"\n+\n" + b"I" * len(long) + b"\n"
    right = b"@a\nACGT\n+\nIIII\n"
    assert fq_ctx.parse_fastq_pairs(left, right).shape[0] == 2
    with pytest.raises(api.HeraGpuError) as e:
        fq_ctx.align_fastq_pairs(left, right, 1)
    assert e.value.code == -4
