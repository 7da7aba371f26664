"""BAM records of the host tail (`-w`): the records align_pair_read appends
per pair (bam_write_pair, src/bam_write.c:382-416), from the `-w` Candidate
records and GENE_MAP.  The oracle's restatement against the reference's own
bytes (golden and live), and the device writer's code
(hera_b200/csrc/hera_bam_core.h) compiled for the host against the golden
bytes; tests/test_tail_classes.py runs the writer on the GPU."""
import json
import multiprocessing as mp
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle
from hera_b200 import index, synth, workloads

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SETS = ["pairs100", "pairs150div", "pairs_mixed", "pairs_n", "pairs_long"]


@pytest.fixture(scope="module")
def small():
    if not os.path.exists(oracle.ORACLE_SO):
        pytest.skip("oracle not built")
    meta = json.load(open(os.path.join(GOLD, "golden.json")))
    p = dict(meta["index"])
    for k in ("exons", "intron"):
        p[k] = tuple(p[k])
    ix = index.build_index(synth.transcriptome(synth.make_annotation(**p)))
    return ix, oracle.Oracle(ix)


class _GM(oracle.GeneMap):
    def __init__(self, d):   # the golden copy of GENE_MAP
        self.chr_len, self.exon_off = d["gm_chr_len"], d["gm_exon_off"]
        self.starts, self.ends, self.chr, self.gene = d["gm_starts"], d["gm_ends"], d["gm_chr"], d["gm_gene"]


def _records(orc, gm, r1, r2):
    res = orc.align_pairs(r1, r2, 0)
    q = [np.full(r1.seq.shape[0] + 1, ord("?"), np.uint8), np.full(r2.seq.shape[0] + 1, ord("?"), np.uint8)]
    return oracle.bam_pairs(gm, res, r1, r2, q, [oracle.read_names(r1.n, 1), oracle.read_names(r1.n, 2)])


@pytest.mark.parametrize("name", SETS)
def test_bam_records_golden(small, name):
    ix, orc = small
    c = np.load(os.path.join(GOLD, "candidates.npz"))
    d = np.load(os.path.join(GOLD, "bam.npz"))
    n = int(d[f"{name}_n"][0])
    r1 = synth.ReadSet(c[f"{name}_r1_seq"], c[f"{name}_r1_off"], c[f"{name}_r1_len"]).subset(np.arange(n))
    r2 = synth.ReadSet(c[f"{name}_r2_seq"], c[f"{name}_r2_off"], c[f"{name}_r2_len"]).subset(np.arange(n))
    got, off = _records(orc, _GM(d), r1, r2)
    want, woff = d[f"{name}_bam"], d[f"{name}_bam_off"]
    bad = [i for i in range(n) if got[off[i]:off[i + 1]].tobytes() != want[woff[i]:woff[i + 1]].tobytes()]
    assert not bad, f"{name}: {len(bad)} pairs' records differ, first {bad[0]}"


# 90 transcripts: the reference reads each transcript's exon count as 4
# bytes into a 2-byte array element (src/bam_write.c:46), so the last one
# writes 2 bytes past the array; with n_trans = 4 (mod 8) those land on the
# heap's bookkeeping and glibc aborts.  Other counts are harmless.
LIVE_ANNOTATION = dict(seed=8, genome_len=400_000, n_genes=40, n_transcripts=90, n_chrom=2)


def _live(d, wl, n, q, host_so=None, lower=False):
    """Child process: the reference loads its own index directory (its
    globals would otherwise outlive this test).  With host_so, the device
    writer's code compiled for the host is held to the same bytes."""
    import ctypes as C
    ann = synth.make_annotation(**LIVE_ANNOTATION)
    tx = synth.transcriptome(ann)
    ix = index.build_index(tx)
    lib = C.CDLL(oracle.REFERENCE_SO)
    lib.refh_bam_setup(os.path.join(d, "idx").encode())
    gm = oracle.GeneMap(os.path.join(d, "idx", "reference.inf"), ix.n_trans)
    r1, r2 = workloads.pairs(wl, ann, tx, n, seed=77)
    if lower:   # lower-case bases, which the front half upper-cases
        for rs in (r1, r2):
            m = np.isin(rs.seq, np.frombuffer(b"ACGT", np.uint8)) & (np.arange(rs.seq.shape[0]) % 3 == 0)
            rs.seq[m] += 32
    a1, a2 = r1.copy(), r2.copy()
    qa = [np.full(a1.seq.shape[0] + 1, ord("?"), np.uint8), np.full(a2.seq.shape[0] + 1, ord("?"), np.uint8)]
    names = [oracle.read_names(n, 1), oracle.read_names(n, 2)]   # alive through the call
    buf = np.zeros(1 << 26, np.uint8)
    off = np.zeros(n + 1, np.uint64)
    rc = lib.refh_bam_pairs(n, *oracle._bam_args(a1, a2, qa, names), C.c_void_p(buf.ctypes.data),
                            C.c_uint64(buf.size), C.c_void_p(off.ctypes.data))
    orc = oracle.Oracle(ix)
    got, goff = _records(orc, gm, r1.copy(), r2.copy())
    bad = [i for i in range(n) if got[goff[i]:goff[i + 1]].tobytes() != buf[off[i]:off[i + 1]].tobytes()]
    bad_host = 0
    if host_so:
        h1, h2 = r1.copy(), r2.copy()
        res = orc.align_pairs(h1.copy(), h2.copy(), 0)   # the writer gets the caller's reads as they were
        hb, hoff, herr = host_records(C.CDLL(host_so), gm, res, h1, h2)
        bad_host = herr + sum(1 for i in range(n) if hb[hoff[i]:hoff[i + 1]].tobytes() != buf[off[i]:off[i + 1]].tobytes())
    sg = synth.gene_map(ann)
    gm_same = all(np.array_equal(getattr(sg, k), getattr(gm, k))
                  for k in ("chr_len", "exon_off", "starts", "ends", "chr", "gene"))
    q.put((rc, int(off[-1]), len(bad), bad_host, gm_same))


@pytest.mark.skipif(not oracle.reference_available() or not os.path.exists(oracle.REF_HERA_BUILD),
                    reason="reference not built here")
@pytest.mark.parametrize("wl,lower", [("config1", False), ("config4", False), ("config4", True)])
def test_bam_records_match_reference(tmp_path, host_writer, wl, lower):
    """Two chromosomes, the config-1 and config-4 read models (the latter
    with unmapped and rescued mates), and lower-case bases: every pair's
    records byte for byte, from the oracle and from the device writer's code
    compiled for the host."""
    ann = synth.make_annotation(**LIVE_ANNOTATION)
    d = str(tmp_path)
    synth.write_genome_fasta(ann, os.path.join(d, "g.fa"))
    synth.write_gtf(ann, os.path.join(d, "g.gtf"))
    shutil.copy(oracle.REF_HERA_BUILD, os.path.join(d, "hera_build"))
    shutil.copy(oracle.REFERENCE_BIN, os.path.join(d, "hera"))
    subprocess.run(["python3", os.path.join(d, "hera_build"), "--fasta", os.path.join(d, "g.fa"), "--gtf",
                    os.path.join(d, "g.gtf"), "--outdir", os.path.join(d, "idx")], check=True, capture_output=True)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_live, args=(d, wl, 2000, q, host_writer._name, lower))
    p.start()
    p.join(timeout=240)
    if p.exitcode is None:
        p.kill()
    assert p.exitcode == 0
    rc, nbytes, bad, bad_host, gm_same = q.get(timeout=10)
    assert rc == 0 and nbytes > 0 and bad == 0 and bad_host == 0 and gm_same


@pytest.fixture(scope="module")
def host_writer(tmp_path_factory):
    """tests/bam_host_check.cpp (the device writer's code on the host)."""
    import ctypes as C
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    so = str(tmp_path_factory.mktemp("bamw") / "bam_host_check.so")
    here = os.path.dirname(os.path.abspath(__file__))
    subprocess.run([gxx, "-O2", "-std=c++17", "-shared", "-fPIC", os.path.join(here, "bam_host_check.cpp"),
                    "-o", so], check=True)
    return C.CDLL(so)


def host_records(lib, gm, res, r1, r2, cap=1 << 26):
    import ctypes as C
    n = r1.n
    q = [np.full(r1.seq.shape[0] + 1, ord("?"), np.uint8), np.full(r2.seq.shape[0] + 1, ord("?"), np.uint8)]
    names = [oracle.read_names(n, 1), oracle.read_names(n, 2)]
    out = np.zeros(cap, np.uint8)
    off = np.zeros(n + 1, np.uint64)
    err = C.c_uint32()
    p = lambda a: C.c_void_p(a.ctypes.data)
    arrs = [np.ascontiguousarray(a, np.uint32) for a in (gm.chr_len, gm.exon_off, gm.starts, gm.ends, gm.chr, gm.gene)]
    lib.bam_host_pairs(C.c_uint32(len(arrs[0])), *[p(a) for a in arrs], p(res.recs), p(res.pos_pool), p(res.p_pool),
                       p(res.op_pool), p(res.miss_pool), n, p(r1.seq), p(r1.off), p(r1.len), p(q[0]), p(names[0]),
                       p(r2.seq), p(r2.off), p(r2.len), p(q[1]), p(names[1]), C.c_int32(names[0].shape[1]),
                       p(out), p(off), C.byref(err))
    return out[:int(off[-1])].copy(), off, err.value


@pytest.mark.parametrize("name", SETS)
def test_device_writer_code_on_host_golden(small, host_writer, name):
    """The writer the kernels run, compiled for the host, gives the
    reference's bytes for every golden pair; the inputs stay unmodified."""
    ix, orc = small
    c = np.load(os.path.join(GOLD, "candidates.npz"))
    d = np.load(os.path.join(GOLD, "bam.npz"))
    n = int(d[f"{name}_n"][0])
    r1 = synth.ReadSet(c[f"{name}_r1_seq"], c[f"{name}_r1_off"], c[f"{name}_r1_len"]).subset(np.arange(n))
    r2 = synth.ReadSet(c[f"{name}_r2_seq"], c[f"{name}_r2_off"], c[f"{name}_r2_len"]).subset(np.arange(n))
    res = orc.align_pairs(r1, r2, 0)
    before = (r1.seq.copy(), r2.seq.copy())
    got, off, err = host_records(host_writer, _GM(d), res, r1, r2)
    assert err == 0
    assert np.array_equal(before[0], r1.seq) and np.array_equal(before[1], r2.seq)
    want, woff = d[f"{name}_bam"], d[f"{name}_bam_off"]
    bad = [i for i in range(n) if got[off[i]:off[i + 1]].tobytes() != want[woff[i]:woff[i + 1]].tobytes()]
    assert not bad, f"{name}: {len(bad)} pairs' records differ, first {bad[0]}"


def test_gene_map_from_annotation_matches_hera_build():
    """synth.gene_map gives the GENE_MAP hera_build's reference.inf holds
    (the golden copy was read from the file hera_build wrote)."""
    meta = json.load(open(os.path.join(GOLD, "golden.json")))
    p = dict(meta["index"])
    for k in ("exons", "intron"):
        p[k] = tuple(p[k])
    gm = synth.gene_map(synth.make_annotation(**p))
    d = np.load(os.path.join(GOLD, "bam.npz"))
    for k in ("chr_len", "exon_off", "starts", "ends", "chr", "gene"):
        assert np.array_equal(getattr(gm, k), d[f"gm_{k}"]), k


def host_records_single(lib, gm, res, rs, cap=1 << 25):
    import ctypes as C
    n = rs.n
    q = np.full(rs.seq.shape[0] + 1, ord("?"), np.uint8)
    names = oracle.read_names(n, 1)
    out = np.zeros(cap, np.uint8)
    off = np.zeros(n + 1, np.uint64)
    err = C.c_uint32()
    p = lambda a: C.c_void_p(a.ctypes.data)
    arrs = [np.ascontiguousarray(a, np.uint32) for a in (gm.chr_len, gm.exon_off, gm.starts, gm.ends, gm.chr, gm.gene)]
    lib.bam_host_single(C.c_uint32(len(arrs[0])), *[p(a) for a in arrs], p(res.recs), p(res.pos_pool),
                        p(res.p_pool), p(res.op_pool), p(res.miss_pool), n, p(rs.seq), p(rs.off), p(rs.len), p(q),
                        p(names), C.c_int32(names.shape[1]), p(out), p(off), C.byref(err))
    return out[:int(off[-1])].copy(), off, err.value


def test_device_writer_code_on_host_single_golden(small, host_writer):
    """Single reads: align_single_read's records (bam_write_single), the
    device writer's code built for the host against the reference's bytes."""
    ix, orc = small
    c = np.load(os.path.join(GOLD, "candidates.npz"))
    d = np.load(os.path.join(GOLD, "bam.npz"))
    n = int(d["single_n"][0])
    rs = synth.ReadSet(c["single_seq"], c["single_off"], c["single_len"]).subset(np.arange(n))
    res = orc.align_single(rs.copy(), 0)
    got, off, err = host_records_single(host_writer, _GM(d), res, rs)
    assert err == 0
    want, woff = d["single_bam"], d["single_bam_off"]
    bad = [i for i in range(n) if got[off[i]:off[i + 1]].tobytes() != want[woff[i]:woff[i + 1]].tobytes()]
    assert not bad, f"{len(bad)} reads' records differ, first {bad[0]}"


def test_bam_single_records_golden(small):
    """The oracle's restatement of the single-read writes against the
    reference's golden bytes."""
    ix, orc = small
    c = np.load(os.path.join(GOLD, "candidates.npz"))
    d = np.load(os.path.join(GOLD, "bam.npz"))
    n = int(d["single_n"][0])
    rs = synth.ReadSet(c["single_seq"], c["single_off"], c["single_len"]).subset(np.arange(n))
    res = orc.align_single(rs, 0)
    q = np.full(rs.seq.shape[0] + 1, ord("?"), np.uint8)
    got, off = oracle.bam_single(_GM(d), res, rs, q, oracle.read_names(n, 1))
    want, woff = d["single_bam"], d["single_bam_off"]
    bad = [i for i in range(n) if got[off[i]:off[i + 1]].tobytes() != want[woff[i]:woff[i + 1]].tobytes()]
    assert not bad, f"{len(bad)} reads' records differ, first {bad[0]}"
