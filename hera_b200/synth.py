"""Seeded synthetic genomes, annotations and read sets.

hera's own inputs are a genome FASTA + GTF, turned into a transcriptome by
``hera_build`` (src/hera_build:119-198: exons of a transcript sorted by start,
concatenated in genomic + orientation, named ``transcript_id:gene_id``), and
FASTQ read files.  This module produces the same objects from a seed so that
every workload is reproducible without any external dataset:

* ``make_annotation``  -- genome, genes of 2..N exons (log-normal exon
  lengths, uniform introns), isoforms by exon skipping;
* ``Transcriptome``    -- the transcript set exactly as ``hera_build`` lays it
  out (same order, names and sequences);
* ``simulate_pairs`` / ``simulate_single`` -- fragments drawn by abundance,
  substitutions and short indels, Phred-30 qualities.

The FASTA/GTF/FASTQ writers exist so the reference program can be run on the
very same data.
"""
from __future__ import annotations

import dataclasses
import os
from typing import List, Optional, Sequence

import numpy as np

_ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)
_COMP = np.zeros(256, dtype=np.uint8)
_COMP[:] = np.arange(256, dtype=np.uint8)
for _a, _b in zip(b"ACGTacgt", b"TGCAtgca"):
    _COMP[_a] = _b


def revcomp(a: np.ndarray) -> np.ndarray:
    """Reverse complement of an ASCII uint8 array (last axis)."""
    return _COMP[a[..., ::-1]]


@dataclasses.dataclass
class Gene:
    gene_id: str
    gene_name: str
    chrom: int
    strand: str
    exons: List[tuple]                 # (start0, end_excl) genomic, sorted
    isoforms: List[List[int]]          # exon index lists, one per transcript


@dataclasses.dataclass
class Annotation:
    chrom_names: List[str]
    chroms: List[np.ndarray]           # ASCII uint8 per chromosome
    genes: List[Gene]                  # in GTF order (chromosome, position)


@dataclasses.dataclass
class Transcriptome:
    names: List[str]                   # "transcript_id:gene_id"
    seq: np.ndarray                    # concatenated ASCII uint8
    length: np.ndarray                 # uint32 per transcript
    find: np.ndarray                   # uint32 exclusive end offsets

    @property
    def n(self) -> int:
        return int(self.length.shape[0])

    def starts(self) -> np.ndarray:
        return (self.find.astype(np.int64) - self.length.astype(np.int64))


def _ids(prefix: str, i: int) -> str:
    s = f"{prefix}{i:0{15 - len(prefix)}d}"
    assert len(s) == 15
    return s


def make_annotation(seed: int, genome_len: int, n_genes: int, n_transcripts: int,
                    n_chrom: int = 1, gc: float = 0.41, exons=(2, 8),
                    exon_median: float = 150.0, exon_sigma: float = 0.5,
                    intron=(200, 5000)) -> Annotation:
    """Genome of uniform i.i.d. bases at the given GC content, genes of
    ``exons`` exons (log-normal lengths) separated by uniform introns, placed
    at random, and ``n_transcripts`` isoforms made by skipping internal exons.
    Gene and transcript ids are 15 characters (hera's gene table skips 16)."""
    rng = np.random.default_rng(seed)
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    per = genome_len // n_chrom
    chroms, names = [], []
    for c in range(n_chrom):
        ln = per if c < n_chrom - 1 else genome_len - per * (n_chrom - 1)
        chroms.append(_ACGT[rng.choice(4, size=ln, p=p).astype(np.uint8)])
        names.append(f"chr{c + 1}")

    genes: List[Gene] = []
    for g in range(n_genes):
        ne = int(rng.integers(exons[0], exons[1] + 1))
        el = np.clip(np.round(rng.lognormal(np.log(exon_median), exon_sigma, ne)), 40, 3000).astype(np.int64)
        il = rng.integers(intron[0], intron[1] + 1, ne - 1).astype(np.int64)
        span = int(el.sum() + il.sum())
        c = int(rng.integers(0, n_chrom))
        clen = chroms[c].shape[0]
        if span >= clen:
            raise ValueError("gene span exceeds chromosome length")
        start = int(rng.integers(0, clen - span))
        ex, cur = [], start
        for k in range(ne):
            ex.append((cur, cur + int(el[k])))
            cur += int(el[k]) + (int(il[k]) if k < ne - 1 else 0)
        genes.append(Gene("", "", c, "+" if rng.random() < 0.5 else "-", ex, [list(range(ne))]))

    # extra isoforms by skipping a non-empty subset of internal exons
    extra = n_transcripts - n_genes
    cand = [i for i, g in enumerate(genes) if len(g.exons) >= 3]
    tries = 0
    while extra > 0 and cand and tries < 50 * n_transcripts:
        tries += 1
        g = genes[cand[int(rng.integers(0, len(cand)))]]
        ne = len(g.exons)
        keep = rng.random(ne - 2) < 0.6
        if keep.all():
            keep[int(rng.integers(0, ne - 2))] = False
        iso = [0] + [k + 1 for k in range(ne - 2) if keep[k]] + [ne - 1]
        if iso in g.isoforms:
            continue
        g.isoforms.append(iso)
        extra -= 1

    genes.sort(key=lambda g: (g.chrom, g.exons[0][0]))
    t = 0
    for gi, g in enumerate(genes):
        g.gene_id = _ids("HGENE", gi + 1)
        g.gene_name = _ids("NAME", gi + 1)
    return Annotation(names, chroms, genes)


def transcriptome(ann: Annotation) -> Transcriptome:
    """Transcripts in the order and form hera_build writes them
    (src/hera_build:160-175): per chromosome, per gene, per transcript,
    exons sorted by start, + orientation, name ``transcript_id:gene_id``."""
    names, parts = [], []
    t = 0
    by_chrom = sorted(range(len(ann.chrom_names)))
    for c in by_chrom:
        for g in ann.genes:
            if g.chrom != c:
                continue
            for iso in g.isoforms:
                t += 1
                names.append(f"{_ids('HTRAN', t)}:{g.gene_id}")
                ex = sorted(g.exons[k] for k in iso)
                parts.append(np.concatenate([ann.chroms[c][a:b] for a, b in ex]))
    length = np.array([x.shape[0] for x in parts], dtype=np.uint32)
    seq = np.concatenate(parts) if parts else np.zeros(0, np.uint8)
    return Transcriptome(names, seq, length, np.cumsum(length, dtype=np.uint64).astype(np.uint32))


@dataclasses.dataclass
class GeneMap:
    """hera's GENE_MAP for an annotation, as hera_build writes it to
    reference.inf and contruct_gene_map reads it (src/bam_write.c:22-57):
    chromosome lengths; per transcript (transcriptome order) its exons as
    0-based inclusive [start, end] genome coordinates sorted by start, its
    chromosome and its gene (numbered in the same order)."""
    chr_len: np.ndarray
    exon_off: np.ndarray
    starts: np.ndarray
    ends: np.ndarray
    chr: np.ndarray
    gene: np.ndarray


def gene_map(ann: Annotation) -> GeneMap:
    starts, ends, off, chrs, genes = [], [], [0], [], []
    g_idx = 0
    for c in sorted(range(len(ann.chrom_names))):
        for g in ann.genes:
            if g.chrom != c:
                continue
            for iso in g.isoforms:
                ex = sorted(g.exons[k] for k in iso)
                starts += [a for a, _ in ex]
                ends += [b - 1 for _, b in ex]
                off.append(off[-1] + len(ex))
                chrs.append(c)
                genes.append(g_idx)
            g_idx += 1
    return GeneMap(np.array([x.shape[0] for x in ann.chroms], np.uint32), np.array(off, np.uint32),
                   np.array(starts, np.uint32), np.array(ends, np.uint32), np.array(chrs, np.uint32),
                   np.array(genes, np.uint32))


def random_transcriptome(seed: int, n: int, mean_len: float = 1800.0, sigma: float = 0.5,
                         gc: float = 0.41, min_len: int = 200) -> Transcriptome:
    """Transcripts drawn directly (no genome): log-normal lengths with the
    given mean.  Used where only the transcriptome matters (index sizing)."""
    rng = np.random.default_rng(seed)
    mu = np.log(mean_len) - sigma * sigma / 2
    length = np.maximum(np.round(rng.lognormal(mu, sigma, n)), min_len).astype(np.uint32)
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    seq = _ACGT[rng.choice(4, size=int(length.sum()), p=p).astype(np.uint8)]
    names = [f"{_ids('HTRAN', i + 1)}:{_ids('HGENE', i + 1)}" for i in range(n)]
    return Transcriptome(names, seq, length, np.cumsum(length, dtype=np.uint64).astype(np.uint32))


def family_transcriptome(seed: int, families=((80, 500),), n_other: int = 40, tail: int = 300,
                         other_len: int = 1500, gc: float = 0.41) -> Transcriptome:
    """Transcripts in paralog families: the members of a family of
    (size, shared) share one `shared`-bp sequence, each followed by a
    `tail`-bp sequence of its own; `n_other` unrelated transcripts follow.
    A read from a shared sequence hits every member of its family, so a
    family larger than a per-read list capacity exercises the long-list
    path."""
    rng = np.random.default_rng(seed)
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])

    def rand(n):
        return _ACGT[rng.choice(4, size=n, p=p).astype(np.uint8)]

    parts = []
    for size, shared in families:
        core = rand(shared)
        parts += [np.concatenate([core, rand(tail)]) for _ in range(size)]
    parts += [rand(other_len) for _ in range(n_other)]
    length = np.array([x.shape[0] for x in parts], np.uint32)
    names = [f"{_ids('HTRAN', i + 1)}:{_ids('HGENE', i + 1)}" for i in range(len(parts))]
    return Transcriptome(names, np.concatenate(parts), length,
                         np.cumsum(length, dtype=np.uint64).astype(np.uint32))


def family_pairs(tx: Transcriptome, n: int, seed: int, shared: int, read_len: int = 100,
                 sub_rate: float = 0.005, mate2_random: bool = False) -> tuple:
    """Pairs whose mate 1 comes from the shared sequence of the first
    family (transcript 0's first `shared` bases), forward strand; mate 2 is
    the reverse complement of a later stretch of the same sequence, or
    random sequence (unmappable: the pair then needs a mate rescue over
    every member of the family)."""
    rng = np.random.default_rng(seed)
    src = tx.seq[:shared]
    m1 = np.empty((n, read_len), np.uint8)
    m2 = np.empty((n, read_len), np.uint8)
    for i in range(n):
        a = int(rng.integers(0, max(1, shared - 2 * read_len)))
        m1[i] = src[a:a + read_len]
        if mate2_random:
            m2[i] = _ACGT[rng.integers(0, 4, read_len)]
        else:
            b = int(rng.integers(a, max(a + 1, shared - read_len)))
            m2[i] = revcomp(src[b:b + read_len])
    _substitute(rng, m1, sub_rate)
    _substitute(rng, m2, sub_rate)
    return _pack_matrix(m1), _pack_matrix(m2)


@dataclasses.dataclass
class ReadSet:
    """Reads packed back to back: read i is seq[off[i]:off[i]+len[i]]."""
    seq: np.ndarray
    off: np.ndarray        # int64
    len: np.ndarray        # int32

    @property
    def n(self) -> int:
        return int(self.len.shape[0])

    def read(self, i: int) -> bytes:
        o = int(self.off[i])
        return self.seq[o:o + int(self.len[i])].tobytes()

    def subset(self, idx) -> "ReadSet":
        idx = np.asarray(idx)
        lens = self.len[idx].astype(np.int32)
        off = np.zeros(idx.shape[0], np.int64)
        off[1:] = np.cumsum(lens[:-1], dtype=np.int64)
        total = int(lens.sum())
        seq = np.empty(total, np.uint8)
        src = np.repeat(self.off[idx], lens) + (np.arange(total) - np.repeat(off, lens))
        seq[:] = self.seq[src]
        return ReadSet(seq, off, lens)

    def copy(self) -> "ReadSet":
        return ReadSet(self.seq.copy(), self.off.copy(), self.len.copy())


def _pack(rows: List[np.ndarray]) -> ReadSet:
    lens = np.array([r.shape[0] for r in rows], dtype=np.int32)
    off = np.zeros(len(rows), np.int64)
    if len(rows):
        off[1:] = np.cumsum(lens[:-1], dtype=np.int64)
    seq = np.concatenate(rows) if rows else np.zeros(0, np.uint8)
    return ReadSet(seq, off, lens)


def _pack_matrix(m: np.ndarray) -> ReadSet:
    n, L = m.shape
    return ReadSet(np.ascontiguousarray(m).reshape(-1), np.arange(n, dtype=np.int64) * L,
                   np.full(n, L, dtype=np.int32))


def _mutate(rng, tmpl: np.ndarray, L: int, indel: float, indel_len) -> np.ndarray:
    """Read of length L from a template (>= L + slack bases) with at least
    one indel event (rate `indel` per base), events placed uniformly."""
    n_ev = max(1, int(rng.binomial(L, indel)))
    pos = np.sort(rng.choice(L, size=min(n_ev, L), replace=False))
    out, i, have = [], 0, 0
    for p in pos:
        take = int(p) - have
        if take > 0:
            out.append(tmpl[i:i + take])
            i += take
            have += take
        k = int(rng.integers(indel_len[0], indel_len[1] + 1))
        if rng.random() < 0.5:   # insertion
            out.append(_ACGT[rng.integers(0, 4, k)])
            have += k
        else:                    # deletion
            i += k
    out.append(tmpl[i:i + max(L - have, 0)])
    r = np.concatenate(out)[:L]
    if r.shape[0] < L:
        r = np.concatenate([r, tmpl[:L - r.shape[0]]])
    return r


def _substitute(rng, m: np.ndarray, rate) -> None:
    """In-place uniform substitutions (to a different base) at `rate`
    (scalar or per-row)."""
    rate = np.asarray(rate, dtype=np.float64)
    if rate.ndim == 1:
        rate = rate[:, None]
    hit = rng.random(m.shape) < rate
    if not hit.any():
        return
    idx = np.nonzero(hit)
    cur = m[idx]
    code = np.searchsorted(_ACGT, cur)
    code = np.where(code > 3, 0, code)
    new = (code + rng.integers(1, 4, code.shape[0])) % 4
    ok = np.isin(cur, _ACGT)
    m[idx] = np.where(ok, _ACGT[new], cur)


def _pick_fragments(rng, tx: Transcriptome, n: int, read_len, frag_mu, frag_sd,
                    abundance_sigma: float, abundance=None):
    length = tx.length.astype(np.int64)
    if abundance is None:
        abundance = rng.lognormal(0.0, abundance_sigma, tx.n)
    rl = np.broadcast_to(np.asarray(read_len, dtype=np.int64), (n,))
    w = abundance * np.maximum(length - 0, 0)
    w = w / w.sum()
    t = rng.choice(tx.n, size=n, p=w)
    flen = np.round(rng.normal(frag_mu, frag_sd, n)).astype(np.int64)
    flen = np.maximum(flen, rl)
    short = length[t] < rl
    while short.any():    # a transcript shorter than its read: draw again
        t[short] = rng.choice(tx.n, size=int(short.sum()), p=w)
        short = length[t] < rl
    flen = np.minimum(flen, length[t])
    start = (rng.random(n) * (length[t] - flen + 1)).astype(np.int64)
    gstart = tx.starts()[t] + start
    return t, gstart, flen, rl


def simulate_pairs(tx: Transcriptome, n: int, seed: int, read_len: int = 100,
                   frag_mu: float = 250.0, frag_sd: float = 25.0,
                   sub_rate=0.005, indel_rate: float = 0.0001, indel_len=(1, 3),
                   abundance_sigma: float = 2.0, abundance=None):
    """Paired reads of a fixed length: read 1 from one fragment end, read 2
    the reverse complement of the other, orientation chosen at random."""
    rng = np.random.default_rng(seed)
    t, gstart, flen, _ = _pick_fragments(rng, tx, n, read_len, frag_mu, frag_sd,
                                         abundance_sigma, abundance)
    L = read_len
    ar = np.arange(L, dtype=np.int64)
    left = tx.seq[gstart[:, None] + ar[None, :]]
    right = revcomp(tx.seq[(gstart + flen - L)[:, None] + ar[None, :]])
    flip = rng.random(n) < 0.5
    r1 = np.where(flip[:, None], right, left)
    r2 = np.where(flip[:, None], left, right)
    if isinstance(sub_rate, tuple):
        rate = rng.uniform(sub_rate[0], sub_rate[1], n)
    else:
        rate = np.asarray(sub_rate, dtype=np.float64)
    if indel_rate > 0:
        ev = rng.random((n, 2)) < 1.0 - (1.0 - indel_rate) ** L
        ends = tx.find.astype(np.int64)[t]
        starts_t = tx.starts()[t]
        for i, m in zip(*np.nonzero(ev)):
            fwd = (m == 0) != bool(flip[i])
            if fwd:
                a = int(gstart[i])
                tm = tx.seq[a:min(a + L + 40, int(ends[i]))]
            else:
                b = int(gstart[i] + flen[i])
                tm = revcomp(tx.seq[max(b - L - 40, int(starts_t[i])):b])
            if tm.shape[0] >= L:
                (r1 if m == 0 else r2)[i] = _mutate(rng, tm, L, indel_rate, indel_len)
    _substitute(rng, r1, rate)
    _substitute(rng, r2, rate)
    return _pack_matrix(r1), _pack_matrix(r2)


def simulate_single(tx: Transcriptome, n: int, seed: int, read_lens=(50, 75, 100, 150),
                    weights=(1, 1, 2, 1), sub_rate=(0.001, 0.02), indel_rate: float = 0.0005,
                    indel_len=(1, 3), abundance_sigma: float = 2.0) -> ReadSet:
    """Single-end reads of mixed length; per-read substitution rate drawn
    uniformly from `sub_rate`."""
    rng = np.random.default_rng(seed)
    w = np.asarray(weights, np.float64)
    rl = np.asarray(read_lens)[rng.choice(len(read_lens), size=n, p=w / w.sum())]
    t, gstart, flen, _ = _pick_fragments(rng, tx, n, rl, 250.0, 25.0, abundance_sigma)
    rows = []
    rates = rng.uniform(sub_rate[0], sub_rate[1], n)
    for i in range(n):
        L = int(rl[i])
        a = int(gstart[i])
        r = tx.seq[a:a + L].copy()
        if rng.random() < 0.5:
            r = revcomp(r)
        rows.append(r)
    rs = _pack(rows)
    hit = rng.random(rs.seq.shape[0]) < np.repeat(rates, rs.len)
    idx = np.nonzero(hit)[0]
    code = np.searchsorted(_ACGT, rs.seq[idx])
    rs.seq[idx] = _ACGT[(code + rng.integers(1, 4, idx.shape[0])) % 4]
    return rs


def simulate_mixed_pairs(tx: Transcriptome, n: int, seed: int, read_lens=(50, 75, 100, 150),
                         weights=(1, 1, 2, 1), sub_rate=(0.001, 0.02),
                         indel_rate: float = 0.0005, indel_len=(1, 3)):
    """Pairs whose length is drawn per pair from `read_lens`, with per-pair
    substitution rates; returned as packed ReadSets."""
    rng = np.random.default_rng(seed)
    w = np.asarray(weights, np.float64)
    rl = np.asarray(read_lens)[rng.choice(len(read_lens), size=n, p=w / w.sum())]
    r1s, r2s = [], []
    for L in read_lens:
        idx = np.nonzero(rl == L)[0]
        if idx.shape[0] == 0:
            continue
        a, b = simulate_pairs(tx, idx.shape[0], int(rng.integers(1 << 31)), read_len=int(L),
                              sub_rate=rng.uniform(sub_rate[0], sub_rate[1], idx.shape[0]),
                              indel_rate=indel_rate, indel_len=indel_len)
        r1s.append((idx, a))
        r2s.append((idx, b))
    rows1 = [None] * n
    rows2 = [None] * n
    for (idx, a), (_, b) in zip(r1s, r2s):
        for j, i in enumerate(idx):
            rows1[i] = a.seq[a.off[j]:a.off[j] + a.len[j]]
            rows2[i] = b.seq[b.off[j]:b.off[j] + b.len[j]]
    return _pack(rows1), _pack(rows2)


def mutated_loci_pairs(ann: Annotation, n: int, seed: int, read_len: int = 150,
                       mut_rate: float = 0.15):
    """Pairs drawn from random genome positions (mostly unannotated) and
    heavily mutated, so they fall through unmapped."""
    rng = np.random.default_rng(seed)
    r1 = np.empty((n, read_len), np.uint8)
    r2 = np.empty((n, read_len), np.uint8)
    for i in range(n):
        c = int(rng.integers(0, len(ann.chroms)))
        ch = ann.chroms[c]
        a = int(rng.integers(0, ch.shape[0] - 400))
        r1[i] = ch[a:a + read_len]
        r2[i] = revcomp(ch[a + 250 - read_len:a + 250])
    _substitute(rng, r1, mut_rate)
    _substitute(rng, r2, mut_rate)
    return _pack_matrix(r1), _pack_matrix(r2)


def concat_pairs(parts: Sequence[tuple], seed: int):
    """Shuffle together several (ReadSet, ReadSet) pair sets."""
    rng = np.random.default_rng(seed)
    rows1, rows2 = [], []
    for a, b in parts:
        for i in range(a.n):
            rows1.append(a.seq[a.off[i]:a.off[i] + a.len[i]])
            rows2.append(b.seq[b.off[i]:b.off[i] + b.len[i]])
    perm = rng.permutation(len(rows1))
    return _pack([rows1[i] for i in perm]), _pack([rows2[i] for i in perm])


# --------------------------------------------------------------------------
# writers (so the reference program can be run on the same data)
# --------------------------------------------------------------------------
def write_genome_fasta(ann: Annotation, path: str, width: int = 60) -> None:
    with open(path, "wb") as f:
        for name, s in zip(ann.chrom_names, ann.chroms):
            f.write(b">" + name.encode() + b"\n")
            b = s.tobytes()
            for i in range(0, len(b), width):
                f.write(b[i:i + width] + b"\n")


def write_gtf(ann: Annotation, path: str) -> None:
    t = 0
    with open(path, "w") as f:
        for g in ann.genes:
            chrom = ann.chrom_names[g.chrom]
            gs = min(a for a, _ in g.exons) + 1
            ge = max(b for _, b in g.exons)
            f.write(f"{chrom}\tsynth\tgene\t{gs}\t{ge}\t.\t{g.strand}\t.\t"
                    f"gene_id \"{g.gene_id}\"; gene_name \"{g.gene_name}\";\n")
            tids = []
            for iso in g.isoforms:
                t += 1
                tids.append((_ids("HTRAN", t), iso))
            for tid, iso in tids:
                ex = sorted(g.exons[k] for k in iso)
                f.write(f"{chrom}\tsynth\ttranscript\t{ex[0][0] + 1}\t{ex[-1][1]}\t.\t{g.strand}\t.\t"
                        f"gene_id \"{g.gene_id}\"; transcript_id \"{tid}\";\n")
                for a, b in ex:
                    f.write(f"{chrom}\tsynth\texon\t{a + 1}\t{b}\t.\t{g.strand}\t.\t"
                            f"gene_id \"{g.gene_id}\"; transcript_id \"{tid}\";\n")


def fastq_bytes(reads: ReadSet, mate: Optional[int] = None, prefix: str = "read", qual: int = 63) -> bytes:
    """The reads as one FASTQ chunk (names prefix<i>[/mate], quality `qual`)."""
    suffix = f"/{mate}" if mate else ""
    seq = reads.seq.tobytes()
    q = bytes([qual]) * (int(reads.len.max()) if reads.n else 0)
    off, ln = reads.off.tolist(), reads.len.tolist()
    parts = []
    for i in range(reads.n):
        o, L = off[i], ln[i]
        parts.append(b"@%s%d%s\n%s\n+\n%s\n" % (prefix.encode(), i, suffix.encode(), seq[o:o + L], q[:L]))
    return b"".join(parts)


def write_fastq(reads: ReadSet, path: str, mate: Optional[int] = None, prefix: str = "read") -> None:
    suffix = f"/{mate}" if mate else ""
    with open(path, "wb") as f:
        for i in range(reads.n):
            s = reads.read(i)
            f.write(b"@%s%d%s\n%s\n+\n%s\n" % (prefix.encode(), i, suffix.encode(), s, b"?" * len(s)))


def write_transcripts_fasta(tx: Transcriptome, path: str) -> None:
    with open(path, "wb") as f:
        st = tx.starts()
        for i, name in enumerate(tx.names):
            f.write(b">" + name.encode() + b"\n")
            f.write(tx.seq[st[i]:st[i] + int(tx.length[i])].tobytes() + b"\n")
