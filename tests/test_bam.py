"""BAM records of the host tail (`-w`), restated in the oracle: the records
align_pair_read appends per pair (bam_write_pair, src/bam_write.c:382-416),
from the `-w` Candidate records and GENE_MAP, against the reference's own
bytes.  The device form of this step is not built yet; these tests pin the
checker it will be held to."""
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
SETS = ["pairs100", "pairs150div", "pairs_mixed", "pairs_n"]


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


def _live(d, wl, n, q):
    """Child process: the reference loads its own index directory (its
    globals would otherwise outlive this test)."""
    import ctypes as C
    ann = synth.make_annotation(**LIVE_ANNOTATION)
    tx = synth.transcriptome(ann)
    ix = index.build_index(tx)
    lib = C.CDLL(oracle.REFERENCE_SO)
    lib.refh_bam_setup(os.path.join(d, "idx").encode())
    gm = oracle.GeneMap(os.path.join(d, "idx", "reference.inf"), ix.n_trans)
    r1, r2 = workloads.pairs(wl, ann, tx, n, seed=77)
    a1, a2 = r1.copy(), r2.copy()
    qa = [np.full(a1.seq.shape[0] + 1, ord("?"), np.uint8), np.full(a2.seq.shape[0] + 1, ord("?"), np.uint8)]
    names = [oracle.read_names(n, 1), oracle.read_names(n, 2)]   # alive through the call
    buf = np.zeros(1 << 26, np.uint8)
    off = np.zeros(n + 1, np.uint64)
    rc = lib.refh_bam_pairs(n, *oracle._bam_args(a1, a2, qa, names), C.c_void_p(buf.ctypes.data),
                            C.c_uint64(buf.size), C.c_void_p(off.ctypes.data))
    got, goff = _records(oracle.Oracle(ix), gm, r1.copy(), r2.copy())
    bad = [i for i in range(n) if got[goff[i]:goff[i + 1]].tobytes() != buf[off[i]:off[i + 1]].tobytes()]
    q.put((rc, int(off[-1]), len(bad)))


@pytest.mark.skipif(not oracle.reference_available() or not os.path.exists("/root/reference/src/hera_build"),
                    reason="reference not built here")
@pytest.mark.parametrize("wl", ["config1", "config4"])
def test_bam_records_match_reference(tmp_path, wl):
    """Two chromosomes, the config-1 and config-4 read models (the latter
    with unmapped and rescued mates): every pair's records byte for byte."""
    ann = synth.make_annotation(**LIVE_ANNOTATION)
    d = str(tmp_path)
    synth.write_genome_fasta(ann, os.path.join(d, "g.fa"))
    synth.write_gtf(ann, os.path.join(d, "g.gtf"))
    shutil.copy("/root/reference/src/hera_build", os.path.join(d, "hera_build"))
    shutil.copy(oracle.REFERENCE_BIN, os.path.join(d, "hera"))
    subprocess.run(["python3", os.path.join(d, "hera_build"), "--fasta", os.path.join(d, "g.fa"), "--gtf",
                    os.path.join(d, "g.gtf"), "--outdir", os.path.join(d, "idx")], check=True, capture_output=True)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_live, args=(d, wl, 2000, q))
    p.start()
    p.join(timeout=240)
    if p.exitcode is None:
        p.kill()
    assert p.exitcode == 0
    rc, nbytes, bad = q.get(timeout=10)
    assert rc == 0 and nbytes > 0 and bad == 0
