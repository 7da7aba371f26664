"""The drop-in inside hera itself: `oracle/_ref/hera_gpu` is the reference
program built from its own sources, unchanged, with its paired-end worker
loop supplied by oracle/dropin/hera_gpu_worker.c (one hera_gpu_align_pairs
call per chunk, then hera's own align_pair_read tail per pair).  Run on the
same index directory and FASTQ files as the unmodified `oracle/_ref/hera`,
`hera quant -t 1` must write the same abundance.tsv and abundance.gene.tsv,
byte for byte, and with -w the same BAM records (compared decompressed: the
BGZF framing follows the chunking of the worker loop).  The index directory
is written by this repository's own writers (index file and reference.inf,
each checked byte for byte against hera_build + hera index in
tests/test_index.py)."""
import gzip
import os
import struct
import subprocess

import pytest

import oracle
from hera_b200 import index, synth, workloads

pytestmark = pytest.mark.gpu

HERA = oracle.REFERENCE_BIN
HERA_GPU = os.path.join(oracle.REF_DIR, "hera_gpu")


def _quant(binary, idx, r1, r2, out, extra=()):
    p = subprocess.run([binary, "quant", "-i", idx, "-1", r1, "-2", r2, "-o", out, "-t", "1", *extra],
                       capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-2000:]
    return p.stderr


def _bam_records(raw: bytes) -> bytes:
    """The record section of a decompressed BAM (the header's text holds the
    command line, which names each program's own path and output)."""
    assert raw[:4] == b"BAM\1"
    (l_text,) = struct.unpack_from("<i", raw, 4)
    o = 8 + l_text
    (n_ref,) = struct.unpack_from("<i", raw, o)
    o += 4
    for _ in range(n_ref):
        (l_name,) = struct.unpack_from("<i", raw, o)
        o += 4 + l_name + 4
    return raw[o:]


@pytest.fixture(scope="module")
def dataset(tmp_path_factory):
    if not (os.path.exists(HERA) and os.path.exists(HERA_GPU)):
        pytest.skip("hera / hera_gpu not built (make -C oracle ref dropin)")
    d = tmp_path_factory.mktemp("dropin")
    ann, tx, ix = workloads.build("config1")
    index.write_index_dir(ann, ix, str(d / "idx"))
    files = {}
    for wl, n, seed in (("config1", 40000, 61), ("config4", 12000, 62)):
        r1, r2 = workloads.pairs(wl, ann, tx, n, seed=seed)
        a, b = str(d / f"{wl}_1.fq"), str(d / f"{wl}_2.fq")
        synth.write_fastq(r1, a, mate=1)
        synth.write_fastq(r2, b, mate=2)
        files[wl] = (a, b)
    return d, files


@pytest.mark.parametrize("wl", ["config1", "config4"])
def test_hera_quant_abundances_identical(dataset, wl):
    d, files = dataset
    r1, r2 = files[wl]
    _quant(HERA, str(d / "idx"), r1, r2, str(d / f"ref_{wl}"))
    err = _quant(HERA_GPU, str(d / "idx"), r1, r2, str(d / f"gpu_{wl}"))
    assert "pairs aligned on the device" in err
    for f in ("abundance.tsv", "abundance.gene.tsv"):
        a = open(d / f"ref_{wl}" / f, "rb").read()
        b = open(d / f"gpu_{wl}" / f, "rb").read()
        assert a == b, f"{wl}: {f} differs"


def test_hera_quant_bam_records_identical(dataset):
    """-w: traceback CIGARs, the tail's BAM records and the abundances."""
    d, files = dataset
    r1, r2 = files["config4"]
    _quant(HERA, str(d / "idx"), r1, r2, str(d / "ref_w"), ("-w",))
    _quant(HERA_GPU, str(d / "idx"), r1, r2, str(d / "gpu_w"), ("-w",))
    bams = [f for f in os.listdir(d / "ref_w") if f.endswith(".bam")]
    assert bams
    for f in bams:
        a = _bam_records(gzip.decompress(open(d / "ref_w" / f, "rb").read()))
        b = _bam_records(gzip.decompress(open(d / "gpu_w" / f, "rb").read()))
        assert len(a) > 100000 and a == b, f"{f}: records differ"
    for f in ("abundance.tsv", "abundance.gene.tsv"):
        assert open(d / "ref_w" / f, "rb").read() == open(d / "gpu_w" / f, "rb").read()
