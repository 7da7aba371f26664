"""hera's k-mer hash index: build, read and write it in the reference layout.

The reference index (src/hash_align.c:1060-1159, loaded at :1169-1234) is a
direct-mapped table of H = 2^27 buckets.  The bucket of a 31-mer id is its
low 27 bits; each bucket is an array of ``Bucket{u64 id; u32 start, end}``
sorted by id, and ``[start, end)`` indexes two parallel occurrence arrays
``pos`` (transcript id) and ``p`` (offset of the k-mer's last base).

Layout facts that fix parity:

* index k-mers mask N to A (``ascii_table[c] & 3``, src/hash_align.c:1082);
* buckets are laid out in (bucket, id) order and occurrence lists follow that
  order, each list in (transcript, offset) order (src/hash_align.c:1070-1095);
* the file is ``n, name_len, len[n], find[n], names, seq, n_bucket[H],
  buckets, n_pos, pos[n_pos], p[n_pos]`` (src/hash_align.c:1130-1159).

``build_index`` reproduces that layout from a ``Transcriptome`` (a stable
sort of every occurrence by (bucket, id)), byte-identical to ``hera index``.
"""
from __future__ import annotations

import dataclasses
import os
from typing import List, Optional

import numpy as np

KMER = 31
HBITS = 27
H = 1 << HBITS
BUCKET_DTYPE = np.dtype([("id", "<u8"), ("start", "<u4"), ("end", "<u4")])

_CODE = np.full(256, 4, dtype=np.uint8)
for _i, _c in enumerate(b"ACGT"):
    _CODE[_c] = _i
    _CODE[_c + 32] = _i


@dataclasses.dataclass
class HeraIndex:
    n_trans: int
    name_len: int
    names: bytes                 # n_trans * name_len, NUL padded
    length: np.ndarray           # uint32
    find: np.ndarray             # uint32 exclusive end offsets
    seq: np.ndarray              # uint8 ASCII, find[-1] bytes
    bucket_n: np.ndarray         # uint32[H] entries per bucket
    buckets: np.ndarray          # BUCKET_DTYPE
    pos: np.ndarray              # uint32
    p: np.ndarray                # uint32

    @property
    def n_pos(self) -> int:
        return int(self.pos.shape[0])

    def bucket_off(self) -> np.ndarray:
        off = np.zeros(H + 1, dtype=np.uint64)
        np.cumsum(self.bucket_n, dtype=np.uint64, out=off[1:])
        return off

    def seq_padded(self, pad: int = 64) -> np.ndarray:
        """Transcript bytes followed by `pad` zero bytes (the suffix DP window
        may run up to 7 bytes past the last transcript)."""
        out = np.zeros(self.seq.shape[0] + pad, dtype=np.uint8)
        out[:self.seq.shape[0]] = self.seq
        return out

    def transcript_name(self, i: int) -> str:
        raw = self.names[i * self.name_len:(i + 1) * self.name_len]
        return raw.split(b"\0", 1)[0].decode()


def _kmer_ids(codes: np.ndarray) -> np.ndarray:
    """id[k] of the 31-mer ending at k (valid for k >= 30), by doubling:
    1+2+4+8+16 = 31 characters combined from shifted windows."""
    c = codes.astype(np.uint64)
    n = c.shape[0]

    def shifted(a, k):
        out = np.zeros_like(a)
        if k < n:
            out[k:] = a[:n - k]
        return out

    w1 = c
    w2 = (shifted(w1, 1) << np.uint64(2)) | w1
    w4 = (shifted(w2, 2) << np.uint64(4)) | w2
    w8 = (shifted(w4, 4) << np.uint64(8)) | w4
    w16 = (shifted(w8, 8) << np.uint64(16)) | w8
    return ((shifted(w16, 15) << np.uint64(30)) | (shifted(w8, 7) << np.uint64(14)) |
            (shifted(w4, 3) << np.uint64(6)) | (shifted(w2, 1) << np.uint64(2)) | w1)


def _occurrences(seq: np.ndarray, length: np.ndarray, find: np.ndarray):
    """All (id, transcript, offset) triples in (transcript, offset) order."""
    codes = _CODE[seq] & np.uint8(3)
    ids = _kmer_ids(codes)
    starts = find.astype(np.int64) - length.astype(np.int64)
    tid = np.repeat(np.arange(length.shape[0], dtype=np.uint32), length.astype(np.int64))
    off = (np.arange(seq.shape[0], dtype=np.int64) - np.repeat(starts, length.astype(np.int64)))
    keep = off >= KMER - 1
    return ids[keep], tid[keep], off[keep].astype(np.uint32)


def _build_index_torch(tx, device: str) -> HeraIndex:
    """Same layout as build_index, computed with torch on a GPU (index
    construction is set-up work, not the hot path)."""
    import torch
    dev = torch.device(device)
    seq = torch.from_numpy(np.ascontiguousarray(tx.seq)).to(dev)
    lut = torch.from_numpy(_CODE & np.uint8(3)).to(dev)
    c = lut[seq.long()].long()
    n = c.shape[0]

    def shifted(a, k):
        out = torch.zeros_like(a)
        if k < n:
            out[k:] = a[:n - k]
        return out

    w1 = c
    w2 = (shifted(w1, 1) << 2) | w1
    w4 = (shifted(w2, 2) << 4) | w2
    w8 = (shifted(w4, 4) << 8) | w4
    w16 = (shifted(w8, 8) << 16) | w8
    ids = ((shifted(w16, 15) << 30) | (shifted(w8, 7) << 14) | (shifted(w4, 3) << 6) |
           (shifted(w2, 1) << 2) | w1)
    del w2, w4, w8, w16, c
    length = torch.from_numpy(tx.length.astype(np.int64)).to(dev)
    starts = torch.cumsum(length, 0) - length
    tid = torch.repeat_interleave(torch.arange(length.shape[0], device=dev), length)
    off = torch.arange(n, device=dev) - starts[tid]
    keep = off >= KMER - 1
    ids, tid, off = ids[keep], tid[keep], off[keep]
    mask = H - 1
    composite = ((ids & mask) << (62 - HBITS)) | (ids >> HBITS)
    del ids
    sc, order = torch.sort(composite, stable=True)
    del composite
    pos = tid[order].to(torch.int32)
    p = off[order].to(torch.int32)
    del tid, off, order
    uk, counts = torch.unique_consecutive(sc, return_counts=True)
    del sc
    first = torch.cumsum(counts, 0) - counts
    uid = ((uk & ((1 << (62 - HBITS)) - 1)) << HBITS) | (uk >> (62 - HBITS))
    bucket_n = torch.bincount(uid & mask, minlength=H).to(torch.int32)
    buckets = np.empty(uk.shape[0], dtype=BUCKET_DTYPE)
    buckets["id"] = uid.cpu().numpy().view(np.uint64)
    buckets["start"] = first.to(torch.int32).cpu().numpy().view(np.uint32)
    buckets["end"] = (first + counts).to(torch.int32).cpu().numpy().view(np.uint32)
    names = [nm.encode() for nm in tx.names]
    name_len = max(len(nm) for nm in names) + 1
    nb = b"".join(nm + b"\0" * (name_len - len(nm)) for nm in names)
    out = HeraIndex(len(names), name_len, nb, tx.length.astype(np.uint32),
                    tx.find.astype(np.uint32), tx.seq.astype(np.uint8),
                    bucket_n.cpu().numpy().view(np.uint32), buckets,
                    pos.cpu().numpy().view(np.uint32), p.cpu().numpy().view(np.uint32))
    del uk, counts, first, uid, bucket_n, pos, p
    torch.cuda.empty_cache()
    return out


def build_index(tx, device: Optional[str] = None) -> HeraIndex:
    """Index a Transcriptome exactly as ``hera index`` would
    (get_ref_seq + construct_hash, src/hash_align.c:1060-1128).
    `device="cuda"` builds it with torch on the GPU (same bytes, faster at
    transcriptome scale)."""
    if device is not None and device.startswith("cuda"):
        return _build_index_torch(tx, device)
    ids, tid, off = _occurrences(tx.seq, tx.length, tx.find)
    mask = np.uint64(H - 1)
    # (bucket, id) order as one 62-bit key: bucket in the high 27 bits
    composite = ((ids & mask) << np.uint64(62 - HBITS)) | (ids >> np.uint64(HBITS))
    order = np.argsort(composite, kind="stable")
    sc = composite[order]
    pos = tid[order]
    p = off[order]
    del composite, ids
    if sc.shape[0]:
        brk = np.empty(sc.shape[0], dtype=bool)
        brk[0] = True
        np.not_equal(sc[1:], sc[:-1], out=brk[1:])
        first = np.nonzero(brk)[0]
    else:
        first = np.zeros(0, dtype=np.int64)
    uk = sc[first]
    counts = np.diff(np.append(first, sc.shape[0])).astype(np.uint32)
    uid = ((uk & np.uint64((1 << (62 - HBITS)) - 1)) << np.uint64(HBITS)) | (uk >> np.uint64(62 - HBITS))
    buckets = np.empty(uk.shape[0], dtype=BUCKET_DTYPE)
    buckets["id"] = uid
    buckets["start"] = first.astype(np.uint32)
    buckets["end"] = (first + counts).astype(np.uint32)
    bucket_n = np.bincount((uid & mask).astype(np.int64), minlength=H).astype(np.uint32)
    names = [n.encode() for n in tx.names]
    name_len = max(len(n) for n in names) + 1
    nb = b"".join(n + b"\0" * (name_len - len(n)) for n in names)
    return HeraIndex(len(names), name_len, nb, tx.length.astype(np.uint32),
                     tx.find.astype(np.uint32), tx.seq.astype(np.uint8),
                     bucket_n, buckets, pos.astype(np.uint32), p.astype(np.uint32))


def write_index(ix: HeraIndex, path: str) -> None:
    """Write the reference's index file (src/hash_align.c:1130-1159)."""
    with open(path, "wb") as f:
        f.write(np.array([ix.n_trans, ix.name_len], dtype=np.uint32).tobytes())
        f.write(ix.length.astype(np.uint32).tobytes())
        f.write(ix.find.astype(np.uint32).tobytes())
        f.write(ix.names)
        f.write(ix.seq.tobytes())
        f.write(ix.bucket_n.astype(np.uint32).tobytes())
        f.write(ix.buckets.tobytes())
        f.write(np.array([ix.n_pos], dtype=np.uint32).tobytes())
        f.write(ix.pos.astype(np.uint32).tobytes())
        f.write(ix.p.astype(np.uint32).tobytes())


def write_reference_inf(ann, path: str) -> None:
    """hera's reference.inf for an annotation written as synth.write_gtf and
    synth.write_genome_fasta write it (the file hera_build makes beside the
    index; hera quant reads it at start-up, init_bam_header and
    contruct_gene_map, src/bam_write.c:22-57, 448-496):
      - the BAM header's reference block, led by its byte count: chromosome
        count, then per chromosome name length, name, sequence length;
      - chromosome names as fixed-width NUL-padded rows and their lengths;
      - gene labels (strand + gene_id + gene_name) as fixed-width rows;
      - per transcript, in index order: exon count, exon starts, exon ends
        (inclusive, 0-based), then every transcript's chromosome and gene."""
    import struct
    from . import synth
    names = [n.encode() for n in ann.chrom_names]
    lens = [int(c.shape[0]) for c in ann.chroms]
    out = bytearray()
    block = 4 + sum(8 + len(n) for n in names)
    out += struct.pack("<II", block, len(names))
    for n, ln in zip(names, lens):
        out += struct.pack("<I", len(n)) + n + struct.pack("<I", ln)
    w = max(len(n) for n in names) + 1
    out += struct.pack("<II", len(names), w)
    for n in names:
        out += n + b"\0" * (w - len(n))
    out += struct.pack(f"<{len(lens)}I", *lens)
    labels = [(g.strand + g.gene_id + g.gene_name).encode() for g in ann.genes]
    w = max(len(x) for x in labels) + 1
    out += struct.pack("<II", len(labels), w)
    for x in labels:
        out += x + b"\0" * (w - len(x))
    gm = synth.gene_map(ann)
    for t in range(len(gm.chr)):
        a, b = int(gm.exon_off[t]), int(gm.exon_off[t + 1])
        out += struct.pack("<I", b - a)
        out += gm.starts[a:b].astype("<u4").tobytes() + gm.ends[a:b].astype("<u4").tobytes()
    out += gm.chr.astype("<u4").tobytes() + gm.gene.astype("<u4").tobytes()
    with open(path, "wb") as f:
        f.write(bytes(out))


def write_index_dir(ann, ix: HeraIndex, directory: str) -> None:
    """The index directory hera quant reads: `index` and `reference.inf`."""
    import os
    os.makedirs(directory, exist_ok=True)
    write_index(ix, os.path.join(directory, "index"))
    write_reference_inf(ann, os.path.join(directory, "reference.inf"))


def read_index(path: str) -> HeraIndex:
    """Read the reference's index file (src/hash_align.c:1195-1234)."""
    with open(path, "rb") as f:
        n, name_len = np.frombuffer(f.read(8), dtype=np.uint32)
        n, name_len = int(n), int(name_len)
        length = np.frombuffer(f.read(4 * n), dtype=np.uint32).copy()
        find = np.frombuffer(f.read(4 * n), dtype=np.uint32).copy()
        names = f.read(n * name_len)
        seq = np.frombuffer(f.read(int(find[-1])), dtype=np.uint8).copy()
        bucket_n = np.frombuffer(f.read(4 * H), dtype=np.uint32).copy()
        nb = int(bucket_n.sum(dtype=np.uint64))
        buckets = np.frombuffer(f.read(16 * nb), dtype=BUCKET_DTYPE).copy()
        n_pos = int(np.frombuffer(f.read(4), dtype=np.uint32)[0])
        pos = np.frombuffer(f.read(4 * n_pos), dtype=np.uint32).copy()
        p = np.frombuffer(f.read(4 * n_pos), dtype=np.uint32).copy()
    return HeraIndex(n, name_len, names, length, find, seq, bucket_n, buckets, pos, p)
