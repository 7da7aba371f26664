"""Synthetic workloads are deterministic and have the configured shapes."""
import numpy as np

from hera_b200 import synth, workloads


def test_annotation_deterministic():
    a = synth.transcriptome(synth.make_annotation(seed=3, genome_len=100_000, n_genes=10, n_transcripts=20))
    b = synth.transcriptome(synth.make_annotation(seed=3, genome_len=100_000, n_genes=10, n_transcripts=20))
    assert a.names == b.names and np.array_equal(a.seq, b.seq)
    assert all(len(n.split(":")[0]) == 15 and len(n.split(":")[1]) == 15 for n in a.names)


def test_pairs_deterministic_and_shaped(config1):
    ann, tx, _ = config1
    a1, a2 = workloads.pairs("config1", ann, tx, 2000, seed=4)
    b1, b2 = workloads.pairs("config1", ann, tx, 2000, seed=4)
    assert np.array_equal(a1.seq, b1.seq) and np.array_equal(a2.seq, b2.seq)
    assert (a1.len == 100).all() and (a2.len == 100).all()
    m1, _ = workloads.pairs("config3", ann, tx, 2000, seed=4)
    assert set(np.unique(m1.len)) <= {50, 75, 100, 150}


def test_interleave_layout(config1):
    ann, tx, _ = config1
    r1, r2 = workloads.pairs("config3", ann, tx, 300, seed=5)
    seq, off, lens = workloads.interleave(r1, r2)
    for i in range(r1.n):
        assert seq[off[2 * i]:off[2 * i] + lens[2 * i]].tobytes() == r1.read(i)
        assert seq[off[2 * i + 1]:off[2 * i + 1] + lens[2 * i + 1]].tobytes() == r2.read(i)
