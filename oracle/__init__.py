"""ctypes bindings to the test-side checkers built by oracle/Makefile.

TEST INFRASTRUCTURE ONLY -- imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the hera_b200 product.

* ``Oracle``    -- oracle/_ref/libhera_oracle.so, the C restatement
                   (hera_oracle.c) of the reference's hot path;
* ``Reference`` -- oracle/_ref/libhera_ref.so, the reference's own sources
                   plus ref_harness.c (only where the reference was built).

Both return results as ``Result`` objects holding the flat record arrays
(the same layout the product returns), which ``canonical()`` turns into
plain tuples for comparison.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(REF_DIR, "libhera_oracle.so")
REFERENCE_SO = os.path.join(REF_DIR, "libhera_ref.so")
REFERENCE_BIN = os.path.join(REF_DIR, "hera")
# the reference's source tree, where the checkers are built from (only in a
# container that holds it; the GPU box uses the prebuilt oracle/_ref files)
REF_SRC = os.environ.get("HERA_REF_SRC", "/root/reference/src")
REF_HERA_BUILD = os.path.join(REF_SRC, "hera_build")

REC_DTYPE = np.dtype([
    ("n", "<i4", (2,)), ("err", "<i4", (2,)), ("pair", "<i4"),
    ("list_off", "<u4", (2,)), ("cig_off", "<u4", (2,)), ("miss_off", "<u4", (2,)),
    ("n_cigar", "<u2", (2,)), ("n_miss", "<u2", (2,)),
])
assert REC_DTYPE.itemsize == 52

CIGAR_CHARS = "MIDNSHP=XB"


class _Index(C.Structure):
    _fields_ = [("n_trans", C.c_uint32), ("len", C.c_void_p), ("find", C.c_void_p),
                ("seq", C.c_void_p), ("bucket_off", C.c_void_p), ("buckets", C.c_void_p),
                ("pos", C.c_void_p), ("p", C.c_void_p)]


class _Result(C.Structure):
    _fields_ = [("recs", C.c_void_p), ("pos_pool", C.c_void_p), ("p_pool", C.c_void_p),
                ("op_pool", C.c_void_p), ("miss_pool", C.c_void_p),
                ("list_cap", C.c_uint64), ("op_cap", C.c_uint64), ("miss_cap", C.c_uint64),
                ("list_used", C.c_uint64), ("op_used", C.c_uint64), ("miss_used", C.c_uint64)]


class _Stats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("lookups", "hits", "probes", "occurrences",
                                           "sw_calls", "sw_cells", "ssw_calls", "ssw_cells")]


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class Result:
    """Flat candidate records plus pools (one record per Candidate)."""

    def __init__(self, n_recs: int, list_cap: int, op_cap: int, miss_cap: int):
        self.recs = np.zeros(n_recs, dtype=REC_DTYPE)
        self.pos_pool = np.zeros(max(list_cap, 1), np.uint32)
        self.p_pool = np.zeros(max(list_cap, 1), np.int32)
        self.op_pool = np.zeros(max(op_cap, 1), np.uint32)
        self.miss_pool = np.zeros(max(miss_cap, 1), np.uint8)
        self.c = _Result(_ptr(self.recs), _ptr(self.pos_pool), _ptr(self.p_pool),
                         _ptr(self.op_pool), _ptr(self.miss_pool),
                         list_cap, op_cap, miss_cap, 0, 0, 0)

    def candidate(self, i: int):
        """(pair, [(n, err, pos list, p list, cigar string, miss bytes)] x 2)."""
        r = self.recs[i]
        out = []
        for s in range(2):
            n = int(r["n"][s])
            lo = int(r["list_off"][s])
            co, nc = int(r["cig_off"][s]), int(r["n_cigar"][s])
            mo, nm = int(r["miss_off"][s]), int(r["n_miss"][s])
            ops = self.op_pool[co:co + nc]
            cig = "".join(f"{int(o) >> 4}{CIGAR_CHARS[int(o) & 15]}" for o in ops)
            out.append((n, int(r["err"][s]), tuple(self.pos_pool[lo:lo + n].tolist()),
                        tuple(self.p_pool[lo:lo + n].tolist()), cig,
                        bytes(self.miss_pool[mo:mo + nm])))
        return (int(r["pair"]), tuple(out))

    def canonical(self, lo: int = 0, hi: Optional[int] = None) -> List[tuple]:
        hi = self.recs.shape[0] if hi is None else hi
        return [self.candidate(i) for i in range(lo, hi)]


def _pool_caps(n_recs: int, total_len: int, scale: int = 1):
    return ((n_recs * 64 + 1024) * scale, (n_recs * 16 + total_len * 2 + 1024) * scale,
            (total_len * 2 + 1024) * scale)


def _run_grown(n_recs: int, total_len: int, run, what: str) -> "Result":
    """run(res) -> status, retried with larger pools while they are too
    small (the lists of reads in large paralog families are long)."""
    for scale in (1, 16, 256):
        res = Result(n_recs, *_pool_caps(n_recs, total_len, scale))
        if run(res) == 0:
            return res
    raise RuntimeError(f"{what} result pools too small")


class ClassTable:
    """The add_class state after a run (src/hash_align.c:1564-1602): classes
    in first-insertion order (XXH32 id, read count, transcript list),
    REF_INF->count per transcript, PAIRED and MEAN_FRAG's sum."""

    def __init__(self, ids, counts, ns, ref_off, ref, tx_count, paired, mean_frag):
        self.ids = np.asarray(ids, dtype=np.uint32)
        self.counts = np.asarray(counts, dtype=np.float64)
        self.ns = np.asarray(ns, dtype=np.uint32)
        self.ref_off = np.asarray(ref_off, dtype=np.uint64)
        self.ref = np.asarray(ref, dtype=np.uint32)
        self.tx_count = np.asarray(tx_count, dtype=np.uint32)
        self.paired = int(paired)
        self.mean_frag = float(mean_frag)

    @property
    def n_classes(self) -> int:
        return len(self.ids)

    def lists(self):
        return [tuple(self.ref[int(o):int(o) + int(n)]) for o, n in zip(self.ref_off, self.ns)]

    def key(self):
        """Everything the EM and the summary read, as plain values."""
        return (tuple(self.ids.tolist()), tuple(self.counts.tolist()), tuple(self.lists()),
                tuple(self.tx_count.tolist()), self.paired, self.mean_frag)


def _em_args(table: ClassTable, ix):
    """ctypes arguments of ho_em after n_trans: len, tx_count, n_classes,
    count, n, ref_off, ref (arrays kept alive on the table)."""
    table._em_keep = [np.ascontiguousarray(ix.length, np.uint32), np.ascontiguousarray(table.tx_count, np.uint32),
                      np.ascontiguousarray(table.counts, np.float64), np.ascontiguousarray(table.ns, np.uint32),
                      np.ascontiguousarray(table.ref_off, np.uint64),
                      np.ascontiguousarray(np.append(table.ref, np.uint32(0)), np.uint32)]
    ln, tx, cnt, ns, offs, ref = table._em_keep
    return [C.c_void_p(_ptr(ln)), C.c_void_p(_ptr(tx)), C.c_uint32(table.n_classes), C.c_void_p(_ptr(cnt)),
            C.c_void_p(_ptr(ns)), C.c_void_p(_ptr(offs)), C.c_void_p(_ptr(ref))]


def em_port(table, length) -> tuple:
    """estimate_count restated (ho_em) over any class table with counts, ns,
    ref_off, ref, tx_count and n_classes, with transcript lengths `length`:
    (grama, overlap, rounds).  No index needed."""
    lib = C.CDLL(ORACLE_SO)
    n = len(length)

    class _Ix:
        pass
    ix = _Ix()
    ix.length = np.ascontiguousarray(length, np.uint32)
    g, o = np.zeros(max(n, 1)), np.zeros(max(n, 1))
    rounds = C.c_uint32()
    a = _em_args(table, ix)
    lib.ho_em(C.c_uint32(n), *a, C.c_void_p(_ptr(g)), C.c_void_p(_ptr(o)), C.byref(rounds))
    return g[:n], o[:n], rounds.value


class GeneMap:
    """GENE_MAP as hera builds it from reference.inf (contruct_gene_map,
    src/bam_write.c:22-57, after init_bam_header's reference block)."""

    def __init__(self, path: str, n_trans: int):
        b = open(path, "rb").read()
        u32 = lambda o, k=1: np.frombuffer(b, np.uint32, k, o)
        o = 4 + int(u32(0)[0])
        n_chr, l_chr = (int(x) for x in u32(o, 2))
        o += 8 + n_chr * l_chr
        self.chr_len = u32(o, n_chr).copy()
        o += 4 * n_chr
        n_gene, l_gene = (int(x) for x in u32(o, 2))
        o += 8 + n_gene * l_gene
        starts, ends, off = [], [], [0]
        for _ in range(n_trans):
            ne = int(u32(o)[0]) & 0xFFFF   # read into an unsigned short
            starts.append(u32(o + 4, ne))
            ends.append(u32(o + 4 + 4 * ne, ne))
            o += 4 + 8 * ne
            off.append(off[-1] + ne)
        self.exon_off = np.array(off, np.uint32)
        self.starts = np.concatenate(starts).astype(np.uint32)
        self.ends = np.concatenate(ends).astype(np.uint32)
        self.chr = u32(o, n_trans).copy()
        self.gene = u32(o + 4 * n_trans, n_trans).copy()

    def c_struct(self):
        return _gene_map_struct(self)


class _GMStruct(C.Structure):
    _fields_ = [("n_chr", C.c_uint32), ("chr_len", C.c_void_p), ("exon_off", C.c_void_p),
                ("starts", C.c_void_p), ("ends", C.c_void_p), ("chr", C.c_void_p), ("gene", C.c_void_p)]


def _gene_map_struct(gm):
    """ho_gene_map over any object with chr_len, exon_off, starts, ends, chr
    and gene arrays (the arrays are kept alive on the struct)."""
    keep = [np.ascontiguousarray(getattr(gm, k), np.uint32)
            for k in ("chr_len", "exon_off", "starts", "ends", "chr", "gene")]
    g = _GMStruct(len(keep[0]), *[_ptr(a) for a in keep])
    g._keep = keep
    return g


def read_names(n: int, mate: int, stride: int = 16) -> np.ndarray:
    """Mutable NUL-padded names r000000/1 ... as the BAM writer expects."""
    a = np.zeros((n, stride), np.uint8)
    for i in range(n):
        s = f"r{i:06d}/{mate}".encode()
        a[i, :len(s)] = np.frombuffer(s, np.uint8)
    return a


def _bam_args(r1, r2, quals, names):
    q1, q2 = quals
    n1, n2 = names
    return [C.c_void_p(_ptr(r1.seq)), C.c_void_p(_ptr(r1.off)), C.c_void_p(_ptr(r1.len)), C.c_void_p(_ptr(q1)),
            C.c_void_p(_ptr(n1)), C.c_void_p(_ptr(r2.seq)), C.c_void_p(_ptr(r2.off)), C.c_void_p(_ptr(r2.len)),
            C.c_void_p(_ptr(q2)), C.c_void_p(_ptr(n2)), C.c_int32(n1.shape[1])]


def bam_pairs(gm: GeneMap, res: "Result", r1, r2, quals, names, cap: int = 1 << 26):
    """ho_bam_pairs: the tail's uncompressed BAM records per pair, from the
    oracle's `-w` records.  Returns (bytes, offsets)."""
    lib = C.CDLL(ORACLE_SO)
    n = r1.n
    out = np.zeros(cap, np.uint8)
    off = np.zeros(n + 1, np.uint64)
    g = _gene_map_struct(gm)
    rc = lib.ho_bam_pairs(C.byref(g), C.c_void_p(_ptr(res.recs)), C.c_void_p(_ptr(res.pos_pool)),
                          C.c_void_p(_ptr(res.p_pool)), C.c_void_p(_ptr(res.op_pool)), C.c_void_p(_ptr(res.miss_pool)),
                          n, *_bam_args(r1, r2, quals, names), C.c_void_p(_ptr(out)), C.c_uint64(cap),
                          C.c_void_p(_ptr(off)))
    if rc != 0:
        raise RuntimeError("BAM output buffer too small")
    return out[:int(off[-1])].copy(), off


def bam_single(gm, res: "Result", rs, qual, names, cap: int = 1 << 25):
    """ho_bam_single: the records align_single_read writes with `-w`, per
    read, from the oracle's `-w` single-read records."""
    lib = C.CDLL(ORACLE_SO)
    n = rs.n
    out = np.zeros(cap, np.uint8)
    off = np.zeros(n + 1, np.uint64)
    g = _gene_map_struct(gm)
    rc = lib.ho_bam_single(C.byref(g), C.c_void_p(_ptr(res.recs)), C.c_void_p(_ptr(res.pos_pool)),
                           C.c_void_p(_ptr(res.p_pool)), C.c_void_p(_ptr(res.op_pool)),
                           C.c_void_p(_ptr(res.miss_pool)), n, C.c_void_p(_ptr(rs.seq)), C.c_void_p(_ptr(rs.off)),
                           C.c_void_p(_ptr(rs.len)), C.c_void_p(_ptr(qual)), C.c_void_p(_ptr(names)),
                           C.c_int32(names.shape[1]), C.c_void_p(_ptr(out)), C.c_uint64(cap), C.c_void_p(_ptr(off)))
    if rc != 0:
        raise RuntimeError("BAM output buffer too small")
    return out[:int(off[-1])].copy(), off


def _export_classes(sizes, export, n_trans: int) -> ClassTable:
    nc, rn = C.c_uint32(), C.c_uint64()
    sizes(C.byref(nc), C.byref(rn))
    nc, rn = nc.value, rn.value
    ids = np.zeros(max(nc, 1), np.uint32)
    counts = np.zeros(max(nc, 1), np.float64)
    ns = np.zeros(max(nc, 1), np.uint32)
    offs = np.zeros(max(nc, 1), np.uint64)
    ref = np.zeros(max(rn, 1), np.uint32)
    tx = np.zeros(max(n_trans, 1), np.uint32)
    paired, mf = C.c_uint32(), C.c_double()
    export(C.c_void_p(_ptr(ids)), C.c_void_p(_ptr(counts)), C.c_void_p(_ptr(ns)), C.c_void_p(_ptr(offs)),
           C.c_void_p(_ptr(ref)), C.c_void_p(_ptr(tx)), C.byref(paired), C.byref(mf))
    return ClassTable(ids[:nc], counts[:nc], ns[:nc], offs[:nc], ref[:rn], tx[:n_trans], paired.value, mf.value)


class Oracle:
    """The C restatement (oracle/hera_oracle.c) bound to one index."""

    def __init__(self, ix, so_path: str = ORACLE_SO):
        self.lib = C.CDLL(so_path)
        self.ix = ix
        self._seq = ix.seq_padded()
        self._boff = ix.bucket_off()
        self._buckets = np.ascontiguousarray(ix.buckets)
        self._len = np.ascontiguousarray(ix.length, dtype=np.uint32)
        self._find = np.ascontiguousarray(ix.find, dtype=np.uint32)
        self._pos = np.ascontiguousarray(ix.pos, dtype=np.uint32)
        self._p = np.ascontiguousarray(ix.p, dtype=np.uint32)
        self.cix = _Index(ix.n_trans, _ptr(self._len), _ptr(self._find), _ptr(self._seq),
                          _ptr(self._boff), _ptr(self._buckets), _ptr(self._pos), _ptr(self._p))
        L = self.lib
        L.ho_align_pairs.restype = C.c_int
        L.ho_align_single.restype = C.c_int
        L.ho_sw_align.restype = C.c_int
        L.ho_ssw_align.restype = C.c_int
        L.ho_get_index.restype = C.c_uint64
        L.ho_hash_get.restype = C.c_uint32

    def align_pairs(self, r1, r2, write_bam: int = 1) -> Result:
        """Front half of align_pair_read for every pair.  r1/r2 are
        synth.ReadSet objects; their sequences are modified in place exactly
        as the reference modifies them (lower-case ACGT become upper-case)."""
        n = r1.n
        return _run_grown(2 * n, int(r1.len.sum() + r2.len.sum()), lambda res: self.lib.ho_align_pairs(
            C.byref(self.cix), write_bam, n,
            C.c_void_p(_ptr(r1.seq)), C.c_void_p(_ptr(r1.off)), C.c_void_p(_ptr(r1.len)),
            C.c_void_p(_ptr(r2.seq)), C.c_void_p(_ptr(r2.off)), C.c_void_p(_ptr(r2.len)),
            C.byref(res.c)), "oracle")

    def align_single(self, rs, write_bam: int = 1) -> Result:
        n = rs.n
        return _run_grown(n, int(rs.len.sum()), lambda res: self.lib.ho_align_single(
            C.byref(self.cix), write_bam, n,
            C.c_void_p(_ptr(rs.seq)), C.c_void_p(_ptr(rs.off)), C.c_void_p(_ptr(rs.len)),
            C.byref(res.c)), "oracle")

    def classes(self, results, paired: bool = True) -> ClassTable:
        """add_class as the host tail calls it, over a sequence of flat
        results (one per batch, in input order), on one class table."""
        L = self.lib
        L.ho_classes_new.restype = C.c_void_p
        L.ho_classes_add.restype = C.c_int
        h = L.ho_classes_new(C.c_uint32(self.ix.n_trans))
        try:
            for res in results:
                n = len(res.recs) // 2 if paired else len(res.recs)
                rc = L.ho_classes_add(C.c_void_p(h), C.c_void_p(_ptr(res.recs)), C.c_void_p(_ptr(res.pos_pool)),
                                      C.c_void_p(_ptr(res.p_pool)), n, 1 if paired else 0)
                if rc != 0:
                    raise RuntimeError("a hit list names a transcript outside the index")
            return _export_classes(lambda a, b: L.ho_classes_sizes(C.c_void_p(h), a, b),
                                   lambda *a: L.ho_classes_export(C.c_void_p(h), *a), self.ix.n_trans)
        finally:
            L.ho_classes_free(C.c_void_p(h))

    def em(self, table: "ClassTable"):
        """estimate_count over a class table: (grama, overlap, rounds)."""
        n = self.ix.n_trans
        g, o = np.zeros(max(n, 1)), np.zeros(max(n, 1))
        rounds = C.c_uint32()
        a = _em_args(table, self.ix)
        self.lib.ho_em(C.c_uint32(n), *a, C.c_void_p(_ptr(g)), C.c_void_p(_ptr(o)), C.byref(rounds))
        return g[:n], o[:n], rounds.value

    def xxh32(self, data: bytes, seed: int = 0) -> int:
        self.lib.ho_xxh32.restype = C.c_uint32
        b = _as_u8(data)
        return int(self.lib.ho_xxh32(C.c_void_p(_ptr(b)), C.c_size_t(len(data)), C.c_uint32(seed)))

    def align_pairs_mt(self, r1, r2, write_bam: int, nthreads: int) -> None:
        self.lib.ho_align_pairs_mt(C.byref(self.cix), write_bam, r1.n,
                                   C.c_void_p(_ptr(r1.seq)), C.c_void_p(_ptr(r1.off)), C.c_void_p(_ptr(r1.len)),
                                   C.c_void_p(_ptr(r2.seq)), C.c_void_p(_ptr(r2.off)), C.c_void_p(_ptr(r2.len)),
                                   nthreads)

    def stats(self) -> dict:
        s = _Stats()
        self.lib.ho_get_stats(C.byref(s))
        return {k: getattr(s, k) for k, _ in _Stats._fields_}

    def sw_align(self, ref: bytes, rstart: int, q: bytes, ref_len: int, qlen: int, err: int,
                 write_bam: int = 0):
        return _unit_sw(self.lib.ho_sw_align, None, ref, rstart, q, ref_len, qlen, err, write_bam)

    def ssw_align(self, ref: bytes, read: bytes):
        return _unit_ssw(self.lib.ho_ssw_align, ref, read)

    def get_index(self, seq: bytes, start: int) -> int:
        b = np.frombuffer(seq, dtype=np.uint8).copy()
        return int(self.lib.ho_get_index(C.c_void_p(_ptr(b)), start))


def _unit_sw(fn, write_bam_first, ref, rstart, q, ref_len, qlen, err, write_bam):
    cap = 4096
    rb = np.frombuffer(ref + b"\0" * 64, dtype=np.uint8).copy()
    qb = np.frombuffer(q + b"\0", dtype=np.uint8).copy()
    ops = np.zeros(cap, np.uint32)
    miss = np.zeros(cap, np.uint8)
    n_ops, n_miss = C.c_int(0), C.c_int(0)
    if write_bam_first is None:
        score = fn(C.c_void_p(_ptr(rb)), C.c_uint32(rstart), C.c_void_p(_ptr(qb)), C.c_uint32(ref_len),
                   C.c_uint32(qlen), C.c_int(err), C.c_int(write_bam), C.c_void_p(_ptr(ops)),
                   C.byref(n_ops), C.c_void_p(_ptr(miss)), C.byref(n_miss), C.c_int(cap))
    else:
        score = fn(C.c_int(write_bam), C.c_void_p(_ptr(rb)), C.c_uint32(rstart), C.c_void_p(_ptr(qb)),
                   C.c_uint32(ref_len), C.c_uint32(qlen), C.c_int(err), C.c_void_p(_ptr(ops)),
                   C.byref(n_ops), C.c_void_p(_ptr(miss)), C.byref(n_miss), C.c_int(cap))
    cig = "".join(f"{int(o) >> 4}{CIGAR_CHARS[int(o) & 15]}" for o in ops[:n_ops.value])
    return score, cig, bytes(miss[:n_miss.value])


def _unit_ssw(fn, ref, read):
    cap = 8192
    rb = np.frombuffer(ref + b"\0" * 8, dtype=np.uint8).copy()
    qb = np.frombuffer(read + b"\0", dtype=np.uint8).copy()
    ops = np.zeros(cap, np.uint32)
    miss = np.zeros(cap, np.uint8)
    n_ops, n_miss, skip = C.c_int(0), C.c_int(0), C.c_int(0)
    score = fn(C.c_void_p(_ptr(rb)), C.c_int32(len(ref)), C.c_void_p(_ptr(qb)), C.c_int32(len(read)),
               C.byref(skip), C.c_void_p(_ptr(ops)), C.byref(n_ops), C.c_void_p(_ptr(miss)),
               C.byref(n_miss), C.c_int(cap))
    cig = "".join(f"{int(o) >> 4}{CIGAR_CHARS[int(o) & 15]}" for o in ops[:n_ops.value])
    return score, skip.value, cig, bytes(miss[:n_miss.value])


def reference_available() -> bool:
    return os.path.exists(REFERENCE_SO)


class Reference:
    """The reference's own code (oracle/_ref/libhera_ref.so).  The reference
    keeps its index in process globals, so one index per process."""

    _lib = None

    def __init__(self, ix=None, index_dir: Optional[str] = None):
        if Reference._lib is None:
            Reference._lib = C.CDLL(REFERENCE_SO)
        self.lib = Reference._lib
        self.lib.refh_sw_align.restype = C.c_int
        self.lib.refh_ssw_align.restype = C.c_int
        if index_dir is not None:
            self.lib.refh_load_index(index_dir.encode())
        elif ix is not None:
            self._keep = [ix.seq_padded(), np.ascontiguousarray(ix.length, dtype=np.uint32),
                          np.ascontiguousarray(ix.find, dtype=np.uint32),
                          np.ascontiguousarray(ix.bucket_n, dtype=np.uint32),
                          np.ascontiguousarray(ix.buckets),
                          np.ascontiguousarray(ix.pos, dtype=np.uint32),
                          np.ascontiguousarray(ix.p, dtype=np.uint32)]
            seq, ln, fd, bn, bk, pos, p = self._keep
            self.lib.refh_set_index(C.c_uint32(ix.n_trans), C.c_uint32(ix.name_len),
                                    C.c_void_p(_ptr(ln)), C.c_void_p(_ptr(fd)), C.c_void_p(_ptr(seq)),
                                    C.c_void_p(_ptr(bn)), C.c_void_p(_ptr(bk)), C.c_void_p(_ptr(pos)),
                                    C.c_void_p(_ptr(p)), C.c_uint32(ix.n_pos))

    def align_pairs(self, r1, r2, write_bam: int = 1) -> Result:
        n = r1.n
        return _run_grown(2 * n, int(r1.len.sum() + r2.len.sum()), lambda res: self.lib.refh_align_pairs(
            write_bam, n,
            C.c_void_p(_ptr(r1.seq)), C.c_void_p(_ptr(r1.off)), C.c_void_p(_ptr(r1.len)),
            C.c_void_p(_ptr(r2.seq)), C.c_void_p(_ptr(r2.off)), C.c_void_p(_ptr(r2.len)),
            C.byref(res.c)), "reference")

    def align_single(self, rs, write_bam: int = 1) -> Result:
        n = rs.n
        return _run_grown(n, int(rs.len.sum()), lambda res: self.lib.refh_align_single(
            write_bam, n,
            C.c_void_p(_ptr(rs.seq)), C.c_void_p(_ptr(rs.off)), C.c_void_p(_ptr(rs.len)),
            C.byref(res.c)), "reference")

    def classes(self, r1, r2=None, n_trans: Optional[int] = None) -> ClassTable:
        """The reference's whole worker per read (align_pair_read, or
        align_single_read when r2 is None) with WRITE_BAM = 1, then its
        add_class state.  Works on copies of the reads."""
        L = self.lib
        s1, o1, l1 = r1.seq.copy(), r1.off, r1.len
        if r2 is not None:
            s2, o2, l2 = r2.seq.copy(), r2.off, r2.len
        else:
            s2, o2, l2 = s1, o1, l1
        L.refh_classes_run(1 if r2 is not None else 0, r1.n,
                           C.c_void_p(_ptr(s1)), C.c_void_p(_ptr(o1)), C.c_void_p(_ptr(l1)),
                           C.c_void_p(_ptr(s2)), C.c_void_p(_ptr(o2)), C.c_void_p(_ptr(l2)))
        return _export_classes(L.refh_classes_sizes, L.refh_classes_export, n_trans)

    def em(self, table: "ClassTable", n_trans: int):
        """The reference's estimate_count over a class table: (grama, overlap)."""
        g, o = np.zeros(max(n_trans, 1)), np.zeros(max(n_trans, 1))
        cnt = np.ascontiguousarray(table.counts, np.float64)
        ns = np.ascontiguousarray(table.ns, np.uint32)
        offs = np.ascontiguousarray(table.ref_off, np.uint64)
        ref = np.ascontiguousarray(np.append(table.ref, np.uint32(0)), np.uint32)
        tx = np.ascontiguousarray(table.tx_count, np.uint32)
        self.lib.refh_em(C.c_uint32(table.n_classes), C.c_void_p(_ptr(cnt)), C.c_void_p(_ptr(ns)),
                         C.c_void_p(_ptr(offs)), C.c_void_p(_ptr(ref)), C.c_void_p(_ptr(tx)),
                         C.c_void_p(_ptr(g)), C.c_void_p(_ptr(o)))
        return g[:n_trans], o[:n_trans]

    def xxh32(self, data: bytes, seed: int = 0) -> int:
        self.lib.refh_xxh32.restype = C.c_uint32
        b = _as_u8(data)
        return int(self.lib.refh_xxh32(C.c_void_p(_ptr(b)), C.c_size_t(len(data)), C.c_uint32(seed)))

    def align_pairs_mt(self, r1, r2, write_bam: int, nthreads: int) -> None:
        self.lib.refh_align_pairs_mt(write_bam, r1.n,
                                     C.c_void_p(_ptr(r1.seq)), C.c_void_p(_ptr(r1.off)), C.c_void_p(_ptr(r1.len)),
                                     C.c_void_p(_ptr(r2.seq)), C.c_void_p(_ptr(r2.off)), C.c_void_p(_ptr(r2.len)),
                                     nthreads)

    def sw_align(self, ref: bytes, rstart: int, q: bytes, ref_len: int, qlen: int, err: int,
                 write_bam: int = 0):
        return _unit_sw(self.lib.refh_sw_align, True, ref, rstart, q, ref_len, qlen, err, write_bam)

    def ssw_align(self, ref: bytes, read: bytes):
        return _unit_ssw(self.lib.refh_ssw_align, ref, read)


# ---- FASTQ chunk parsing -----------------------------------------------------

FQ_DTYPE = np.dtype([("name", "<i8"), ("seq", "<i8"), ("qual", "<i8"),
                     ("name_len", "<i4"), ("len", "<i4")])
assert FQ_DTYPE.itemsize == 32


def _as_u8(b) -> np.ndarray:
    return np.frombuffer(bytes(b), np.uint8)


def parse_fq_pairs(left: bytes, right: bytes, cap: Optional[int] = None):
    """The restatement (hera_oracle.c): (status, recs[2n], n_pairs, bad_file,
    bad_rec); status 0 ok, -1 READ_FAIL, -2 over cap."""
    lib = C.CDLL(ORACLE_SO)
    lb, rb = _as_u8(left), _as_u8(right)
    if cap is None:
        cap = max(1, (lb.size + rb.size) // 8 + 1)
    out = np.zeros(2 * cap, FQ_DTYPE)
    n, bf, br = C.c_int32(0), C.c_int32(0), C.c_int64(0)
    rc = lib.ho_parse_fq_pairs(C.c_void_p(_ptr(lb)), C.c_int64(lb.size), C.c_void_p(_ptr(rb)),
                               C.c_int64(rb.size), C.c_void_p(_ptr(out)), C.c_int32(cap),
                               C.byref(n), C.byref(bf), C.byref(br))
    return rc, out[:2 * min(n.value, cap)], n.value, bf.value, br.value


def parse_fq_single(buf: bytes, cap: Optional[int] = None):
    lib = C.CDLL(ORACLE_SO)
    b = _as_u8(buf)
    if cap is None:
        cap = max(1, b.size // 4 + 1)
    out = np.zeros(cap, FQ_DTYPE)
    n, br = C.c_int32(0), C.c_int64(0)
    rc = lib.ho_parse_fq_single(C.c_void_p(_ptr(b)), C.c_int64(b.size), C.c_void_p(_ptr(out)),
                                C.c_int32(cap), C.byref(n), C.byref(br))
    return rc, out[:min(n.value, cap)], n.value, 0, br.value


def _nul_copy(b: bytes) -> np.ndarray:
    a = np.zeros(len(b) + 1, np.uint8)
    a[:len(b)] = np.frombuffer(bytes(b), np.uint8)
    return a


def _recs_from_i64(a: np.ndarray, n: int) -> np.ndarray:
    a = a[:5 * n].reshape(n, 5)
    out = np.zeros(n, FQ_DTYPE)
    for k, f in enumerate(("name", "seq", "qual", "name_len", "len")):
        out[f] = a[:, k]
    return out


def ref_parse_fq_pairs(left: bytes, right: bytes, buffers: Optional[list] = None):
    """The reference's get_read_from_fq_buffer in align_pool_pair's loop
    (oracle/_ref/libhera_ref.so); same return form as parse_fq_pairs.
    `buffers`, if given, receives the two buffers as the reader left them."""
    lib = C.CDLL(REFERENCE_SO)
    lb, rb = _nul_copy(left), _nul_copy(right)
    cap = max(1, (lb.size + rb.size) // 8 + 1)
    rec = np.zeros(10 * cap, np.int64)
    n, bf, br = C.c_int32(0), C.c_int32(0), C.c_int64(0)
    rc = lib.refh_parse_fq_pairs(C.c_void_p(_ptr(lb)), C.c_void_p(_ptr(rb)), C.c_void_p(_ptr(rec)),
                                 C.c_int32(cap), C.byref(n), C.byref(bf), C.byref(br))
    m = min(n.value, cap)
    if buffers is not None:
        buffers[:] = [lb[:-1].tobytes(), rb[:-1].tobytes()]
    return rc, _recs_from_i64(rec, 2 * m), n.value, bf.value, br.value


def ref_parse_fq_single(buf: bytes):
    lib = C.CDLL(REFERENCE_SO)
    b = _nul_copy(buf)
    cap = max(1, b.size // 4 + 1)
    rec = np.zeros(5 * cap, np.int64)
    n, br = C.c_int32(0), C.c_int64(0)
    rc = lib.refh_parse_fq_single(C.c_void_p(_ptr(b)), C.c_void_p(_ptr(rec)), C.c_int32(cap),
                                  C.byref(n), C.byref(br))
    return rc, _recs_from_i64(rec, min(n.value, cap)), n.value, 0, br.value
