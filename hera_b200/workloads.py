"""Named synthetic workloads (the shapes of the benchmark configurations).

config1  small transcriptome: 2 Mbp genome (GC 0.41), 200 genes of 2-8
         exons (log-normal, median 150 bp), introns 200-5000 bp, 500
         isoforms by exon skipping; 2x100 bp pairs, fragments N(250, 25),
         log-normal(sigma 2) abundances, 0.5% substitutions, 0.01% 1-3 bp
         indels.
config2  transcriptome scale: 400 Mbp genome in 8 chromosomes, 60k genes,
         200k transcripts (352 Mbp transcriptome, 1.76 kb mean); 2x100 bp
         pairs, 0.5% substitutions, 0.02% indels; 1M-pair chunks.
config2s config 2's gene and read model on a 40 Mbp genome (6k genes,
         20k transcripts): the profiling case.
config3  config1 index; mixed 50/75/100/150 bp reads (1:1:2:1), half paired
         and half single-end, per-read substitution rate U(0.1%, 2%),
         0.05% indels.
config4  config1 index; 2x150 bp, 3% substitutions, 0.5% 1-8 bp indels,
         plus 5% pairs from mutated unannotated loci.

All data is generated from fixed seeds (no external dataset).
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from . import index as _index
from . import synth

ANNOTATIONS = {
    "config1": dict(seed=1, genome_len=2_000_000, n_genes=200, n_transcripts=500, n_chrom=1,
                    exons=(2, 8), exon_median=150.0, intron=(200, 5000)),
    "config2": dict(seed=2, genome_len=400_000_000, n_genes=60_000, n_transcripts=200_000,
                    n_chrom=8, exons=(2, 16), exon_median=208.0, intron=(200, 3000)),
}
# config 2's gene and read model on a tenth of the genome (profiling case:
# same isoform structure, ~1 GB of index on the device)
ANNOTATIONS["config2s"] = dict(seed=2, genome_len=40_000_000, n_genes=6_000, n_transcripts=20_000,
                               n_chrom=2, exons=(2, 16), exon_median=208.0, intron=(200, 3000))
ANNOTATIONS["config3"] = ANNOTATIONS["config1"]
ANNOTATIONS["config4"] = ANNOTATIONS["config1"]

DESCRIPTION = {
    "config1": "2 Mbp genome, 200 genes, 500 isoforms; 2x100 bp, 0.5% subs, 0.01% indels",
    "config2": "400 Mbp genome, 60k genes, 200k transcripts (352 Mbp, 1.76 kb mean); 2x100 bp, "
               "0.5% subs, 0.02% indels",
    "config2s": "40 Mbp genome, 6k genes, 20k transcripts; config-2 read model",
    "config3": "config1 index; 50/75/100/150 bp mixed, U(0.1-2%) subs, 0.05% indels",
    "config4": "config1 index; 2x150 bp, 3% subs, 0.5% 1-8 bp indels, 5% mutated loci",
}


def annotation(name: str) -> synth.Annotation:
    return synth.make_annotation(**ANNOTATIONS[name])


def build(name: str, device: Optional[str] = None):
    """(annotation, transcriptome, index) of a workload."""
    ann = annotation(name)
    tx = synth.transcriptome(ann)
    ix = _index.build_index(tx, device=device)
    return ann, tx, ix


def pairs(name: str, ann, tx, n: int, seed: int):
    """`n` read pairs of the workload's read model."""
    if name == "config1":
        return synth.simulate_pairs(tx, n, seed, read_len=100, sub_rate=0.005,
                                    indel_rate=0.0001, indel_len=(1, 3))
    if name in ("config2", "config2s"):
        return synth.simulate_pairs(tx, n, seed, read_len=100, sub_rate=0.005,
                                    indel_rate=0.0002, indel_len=(1, 3))
    if name == "config3":
        return synth.simulate_mixed_pairs(tx, n, seed, sub_rate=(0.001, 0.02),
                                          indel_rate=0.0005)
    if name == "config4":
        n_mut = n // 20
        a = synth.simulate_pairs(tx, n - n_mut, seed, read_len=150, frag_mu=300.0, frag_sd=30.0,
                                 sub_rate=0.03, indel_rate=0.005, indel_len=(1, 8))
        b = synth.mutated_loci_pairs(ann, n_mut, seed + 1, read_len=150)
        return synth.concat_pairs([a, b], seed + 2)
    raise KeyError(name)


def singles(name: str, tx, n: int, seed: int) -> synth.ReadSet:
    if name == "config3":
        return synth.simulate_single(tx, n, seed, sub_rate=(0.001, 0.02), indel_rate=0.0005)
    return synth.simulate_single(tx, n, seed, read_lens=(100,), weights=(1,), sub_rate=(0.005, 0.005))


def interleave(r1: synth.ReadSet, r2: synth.ReadSet):
    """Mates interleaved (read 2i = mate 1, 2i+1 = mate 2) as one packed
    set, the layout of the device-resident entry point."""
    n = r1.n
    lens = np.empty(2 * n, np.int32)
    lens[0::2] = r1.len
    lens[1::2] = r2.len
    off = np.zeros(2 * n, np.int64)
    off[1:] = np.cumsum(lens[:-1], dtype=np.int64)
    seq = np.empty(int(lens.sum()), np.uint8)
    if np.all(r1.len == r1.len[0]) and np.all(r2.len == r1.len[0]):
        L = int(r1.len[0])
        m = np.empty((n, 2, L), np.uint8)
        m[:, 0, :] = r1.seq.reshape(n, L)
        m[:, 1, :] = r2.seq.reshape(n, L)
        seq[:] = m.reshape(-1)
    else:
        for i in range(n):
            seq[off[2 * i]:off[2 * i] + lens[2 * i]] = r1.seq[r1.off[i]:r1.off[i] + r1.len[i]]
            seq[off[2 * i + 1]:off[2 * i + 1] + lens[2 * i + 1]] = r2.seq[r2.off[i]:r2.off[i] + r2.len[i]]
    return seq, off, lens
