"""The tail's BAM records (`-w`) on the device (hera_gpu_bam_pairs,
hera_gpu_bam_single): the reads aligned on the device with traceback, then
their records written on the device, against the bytes the reference's own
align_pair_read / align_single_read wrote for the same reads
(tests/golden/bam.npz)."""
import json
import os

import numpy as np
import pytest

import oracle
from hera_b200 import api, index, synth

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SETS = ["pairs100", "pairs150div", "pairs_mixed", "pairs_n"]


class _GM:
    def __init__(self, d):
        self.chr_len, self.exon_off = d["gm_chr_len"], d["gm_exon_off"]
        self.starts, self.ends, self.chr, self.gene = d["gm_starts"], d["gm_ends"], d["gm_chr"], d["gm_gene"]


@pytest.fixture(scope="module")
def writer():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    meta = json.load(open(os.path.join(GOLD, "golden.json")))
    prm = dict(meta["index"])
    for k in ("exons", "intron"):
        prm[k] = tuple(prm[k])
    ix = index.build_index(synth.transcriptome(synth.make_annotation(**prm)))
    ctx = api.Context(ix)
    w = api.BamWriter(ctx, _GM(np.load(os.path.join(GOLD, "bam.npz"))))
    yield ctx, w
    w.close()
    ctx.close()


@pytest.mark.parametrize("name", SETS)
def test_device_bam_records_golden(writer, name):
    ctx, w = writer
    c = np.load(os.path.join(GOLD, "candidates.npz"))
    d = np.load(os.path.join(GOLD, "bam.npz"))
    n = int(d[f"{name}_n"][0])
    r1 = synth.ReadSet(c[f"{name}_r1_seq"], c[f"{name}_r1_off"], c[f"{name}_r1_len"]).subset(np.arange(n))
    r2 = synth.ReadSet(c[f"{name}_r2_seq"], c[f"{name}_r2_off"], c[f"{name}_r2_len"]).subset(np.arange(n))
    res = ctx.align_pairs(r1, r2, 0)
    q1 = np.full(r1.seq.shape[0] + 1, ord("?"), np.uint8)
    q2 = np.full(r2.seq.shape[0] + 1, ord("?"), np.uint8)
    got, off, ms = w.pairs(res, r1, r2, q1, q2, oracle.read_names(n, 1), oracle.read_names(n, 2))
    want, woff = d[f"{name}_bam"], d[f"{name}_bam_off"]
    bad = [i for i in range(n) if got[off[i]:off[i + 1]].tobytes() != want[woff[i]:woff[i + 1]].tobytes()]
    assert not bad, f"{name}: {len(bad)} pairs' records differ, first {bad[0]}"
    assert ms > 0


def test_device_bam_single_records_golden(writer):
    """The 800 golden single reads: align_single_read's records."""
    ctx, w = writer
    c = np.load(os.path.join(GOLD, "candidates.npz"))
    d = np.load(os.path.join(GOLD, "bam.npz"))
    n = int(d["single_n"][0])
    rs = synth.ReadSet(c["single_seq"], c["single_off"], c["single_len"]).subset(np.arange(n))
    res = ctx.align_single(rs, 0)
    q = np.full(rs.seq.shape[0] + 1, ord("?"), np.uint8)
    got, off, ms = w.single(res, rs, q, oracle.read_names(n, 1))
    want, woff = d["single_bam"], d["single_bam_off"]
    bad = [i for i in range(n) if got[off[i]:off[i + 1]].tobytes() != want[woff[i]:woff[i + 1]].tobytes()]
    assert not bad, f"{len(bad)} reads' records differ, first {bad[0]}"
    assert n >= 800 and ms > 0


def test_device_bgzf_decompresses_to_input(writer):
    """BGZF on the device (hera_gpu_bgzf): the golden BAM records of every
    set, random and constant buffers, and sizes at the block boundary; each
    result a valid BGZF stream that decompresses to its input, and the
    records' stream at most half their size."""
    import gzip
    import struct
    ctx, _ = writer
    d = np.load(os.path.join(GOLD, "bam.npz"))
    rng = np.random.default_rng(9)
    recs = b"".join(d[f"{k}_bam"].tobytes() for k in SETS)
    cases = [recs, rng.integers(0, 256, 300_000, dtype=np.uint8).tobytes(), b"Q" * 0xff00, b"Q" * (0xff00 + 1),
             b"ACGT", recs * 9]
    for data in cases:
        z, ms = ctx.bgzf(data)
        z = z.tobytes()
        o, blocks = 0, 0
        while o < len(z):
            assert z[o:o + 4] == b"\x1f\x8b\x08\x04" and z[o + 12:o + 16] == b"BC\x02\x00"
            o += struct.unpack_from("<H", z, o + 16)[0] + 1
            blocks += 1
        assert o == len(z) and blocks == -(-len(data) // 0xff00)
        assert gzip.decompress(z) == data
    z, _ = ctx.bgzf(recs)
    assert len(z) < len(recs) / 2
