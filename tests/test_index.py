"""Index builders: numpy, torch and hera's own `hera index` agree byte for
byte; the index file round-trips."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle
from hera_b200 import index, synth

FIELDS = ("names", "length", "find", "seq", "bucket_n", "buckets", "pos", "p")


def _same(a, b):
    for f in FIELDS:
        x, y = getattr(a, f), getattr(b, f)
        assert (x == y) if isinstance(x, bytes) else np.array_equal(x, y), f


def test_torch_builder_matches_numpy():
    ann = synth.make_annotation(seed=5, genome_len=200_000, n_genes=20, n_transcripts=50)
    tx = synth.transcriptome(ann)
    _same(index.build_index(tx), index._build_index_torch(tx, "cpu"))


def test_index_file_round_trip(tmp_path, config1):
    ix = config1[2]
    path = str(tmp_path / "index")
    index.write_index(ix, path)
    _same(ix, index.read_index(path))


@pytest.mark.skipif(not os.path.exists(oracle.REF_HERA_BUILD) or
                    not os.path.exists(oracle.REFERENCE_BIN), reason="reference not available")
def test_matches_hera_index(tmp_path):
    """hera_build + `hera index` on the same genome/GTF give the same bytes."""
    ann = synth.make_annotation(seed=6, genome_len=300_000, n_genes=30, n_transcripts=75, n_chrom=2)
    d = tmp_path
    synth.write_genome_fasta(ann, str(d / "g.fa"))
    synth.write_gtf(ann, str(d / "g.gtf"))
    shutil.copy(oracle.REF_HERA_BUILD, d / "hera_build")
    shutil.copy(oracle.REFERENCE_BIN, d / "hera")
    r = subprocess.run(["python3", str(d / "hera_build"), "--fasta", str(d / "g.fa"), "--gtf",
                        str(d / "g.gtf"), "--outdir", str(d / "idx")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    mine = index.build_index(synth.transcriptome(ann))
    index.write_index(mine, str(d / "mine"))
    assert open(d / "mine", "rb").read() == open(d / "idx" / "index", "rb").read()
    index.write_reference_inf(ann, str(d / "mine.inf"))
    assert open(d / "mine.inf", "rb").read() == open(d / "idx" / "reference.inf", "rb").read()
