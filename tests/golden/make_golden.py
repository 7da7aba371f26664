#!/usr/bin/env python
"""Generate the golden vectors in this directory from the reference program.

    make -C oracle && python tests/golden/make_golden.py

Every expected value here is produced by the reference's own code
(oracle/_ref/libhera_ref.so, the reference sources compiled unchanged by
oracle/Makefile): SW_align and ssw_align called directly, and the front
half of align_pair_read / align_single_read run over reads of a small
seeded synthetic index.  The inputs are seeded synthetic data; the index is
regenerated from its seed by the tests (its digest is stored to catch
generator drift).
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hera_b200 import index, synth  # noqa: E402
import oracle  # noqa: E402

SMALL = dict(seed=11, genome_len=300_000, n_genes=30, n_transcripts=75, n_chrom=1,
             exons=(2, 8), exon_median=150.0, intron=(200, 3000))


def index_digest(ix) -> str:
    h = hashlib.sha256()
    for a in (ix.length, ix.find, ix.seq, ix.bucket_n, ix.buckets, ix.pos, ix.p):
        h.update(np.ascontiguousarray(a).tobytes())
    h.update(ix.names)
    return h.hexdigest()


def small_index():
    ann = synth.make_annotation(**SMALL)
    tx = synth.transcriptome(ann)
    return ann, tx, index.build_index(tx)


A = np.frombuffer(b"ACGT", np.uint8)


def mutate(rng, s: bytes, rate: float) -> bytes:
    out = bytearray()
    for c in s:
        r = rng.random()
        if r < rate / 3:
            out.append(int(A[rng.integers(0, 4)]))
        elif r < 2 * rate / 3:
            pass
        elif r < rate:
            out += bytes([c, int(A[rng.integers(0, 4)])])
        else:
            out.append(c)
    return bytes(out)


def sw_cases(rng, n):
    """SW_align inputs of the live domain (ref_len >= len), both error caps
    and prefix (negative err) form, gaps 0..70 plus ragged edges."""
    cases = []
    for _ in range(n):
        ql = int(rng.integers(0, 71))
        kind = rng.integers(0, 3)
        if kind == 0:       # suffix gap: ref_len = len + 7
            rl = ql + 7
            err = 3 if ql < 14 else 7
        elif kind == 1:     # middle gap: ref_len = len
            rl = ql
            err = 3 if ql < 14 else 7
        else:               # prefix: ref_len = len + add, err negative
            rl = ql + int(rng.integers(0, 8))
            err = -3 if ql < 14 else -7
        base = bytes(A[rng.integers(0, 4, rl + 12)])
        q = mutate(rng, base[:max(ql, 1)], float(rng.random()) * 0.35)[:ql]
        if len(q) < ql:
            q += bytes(A[rng.integers(0, 4, ql - len(q))])
        if rng.random() < 0.05 and ql:
            q = bytes(c if rng.random() > 0.1 else ord("N") for c in q)
        cases.append((base[:rl], q, rl, ql, err))
    return cases


def ssw_cases(rng, n):
    cases = []
    for _ in range(n):
        L = int(rng.choice([20, 50, 75, 100, 150, 253, 260, 300]))
        rl = int(rng.integers(1, 1001))
        ref = bytes(A[rng.integers(0, 4, rl)])
        if rng.random() < 0.7 and rl > L:
            st = int(rng.integers(0, rl - L + 1))
            read = mutate(rng, ref[st:st + L], float(rng.random()) * 0.12)[:L]
            if len(read) < L:
                read += bytes(A[rng.integers(0, 4, L - len(read))])
        else:
            read = bytes(A[rng.integers(0, 4, L)])
        if rng.random() < 0.15:
            read = bytes(c if rng.random() > 0.05 else ord("N") for c in read)
        cases.append((ref, read))
    return cases


def pack_strs(items):
    off = np.zeros(len(items) + 1, np.int64)
    off[1:] = np.cumsum([len(x) for x in items])
    return np.frombuffer(b"".join(items), np.uint8).copy() if items else np.zeros(0, np.uint8), off


def records_to_arrays(res):
    return {"recs": res.recs, "pos": res.pos_pool[:res.c.list_used], "p": res.p_pool[:res.c.list_used],
            "ops": res.op_pool[:res.c.op_used], "miss": res.miss_pool[:res.c.miss_used]}


def main():
    if not oracle.reference_available():
        sys.exit("reference not built: make -C oracle")
    rng = np.random.default_rng(2024)
    ann, tx, ix = small_index()
    ref = oracle.Reference(ix)
    meta = {"index": SMALL, "index_digest": index_digest(ix)}

    # --- SW_align ---
    cases = sw_cases(rng, 3000)
    refs, roff = pack_strs([c[0] for c in cases])
    qs, qoff = pack_strs([c[1] for c in cases])
    out = {"ref": refs, "ref_off": roff, "q": qs, "q_off": qoff,
           "err": np.array([c[4] for c in cases], np.int32)}
    for wb in (1, 0):
        sc, cig, miss = [], [], []
        for r, q, rl, ql, err in cases:
            s, c, m = ref.sw_align(r + b"\0" * 16, 0, q, rl, ql, err, wb)
            sc.append(s)
            cig.append(c.encode())
            miss.append(m)
        out[f"score_wb{wb}"] = np.array(sc, np.int32)
        out[f"cigar_wb{wb}"], out[f"cigar_off_wb{wb}"] = pack_strs(cig)
        out[f"miss_wb{wb}"], out[f"miss_off_wb{wb}"] = pack_strs(miss)
    np.savez_compressed(os.path.join(HERE, "sw_align.npz"), **out)

    # --- ssw_align ---
    cases = ssw_cases(rng, 600)
    refs, roff = pack_strs([c[0] for c in cases])
    reads, doff = pack_strs([c[1] for c in cases])
    sc, sk, cig, miss = [], [], [], []
    for r, d in cases:
        s, k, c, m = ref.ssw_align(r, d)
        sc.append(s)
        sk.append(k)
        cig.append(c.encode())
        miss.append(m)
    cg, cgo = pack_strs(cig)
    ms, mso = pack_strs(miss)
    np.savez_compressed(os.path.join(HERE, "ssw_align.npz"), ref=refs, ref_off=roff, read=reads,
                        read_off=doff, score=np.array(sc, np.int32), skip=np.array(sk, np.int32),
                        cigar=cg, cigar_off=cgo, miss=ms, miss_off=mso)

    # --- k-mer ids (get_index), N bleeding into the neighbour's field ---
    kms = []
    for _ in range(200):
        s = bytes(A[rng.integers(0, 4, 31)])
        if rng.random() < 0.5:
            s = bytes(c if rng.random() > 0.1 else ord("N") for c in s)
        kms.append(s)
    import ctypes as C
    ref.lib.get_index.restype = C.c_ulong
    ref.lib.get_index.argtypes = [C.c_uint, C.c_char_p]
    ids = [ref.lib.get_index(0, k) for k in kms]
    ref.lib.hash_get.restype = C.c_uint
    ref.lib.hash_get.argtypes = [C.c_ulong, C.POINTER(C.c_uint), C.c_uint]
    # probes of the index: ids of real k-mers (hits) and of the random ones
    probe_ids = [int(x) for x in ix.buckets["id"][rng.integers(0, ix.buckets.shape[0], 300)]] + ids
    found, slot = [], []
    for pid in probe_ids:
        ret = C.c_uint(0)
        slot.append(ref.lib.hash_get(pid, C.byref(ret), 0))
        found.append(ret.value)
    np.savez_compressed(os.path.join(HERE, "kmers.npz"),
                        kmer=np.frombuffer(b"".join(kms), np.uint8),
                        ids=np.array(ids, np.uint64),
                        probe_ids=np.array(probe_ids, np.uint64),
                        probe_found=np.array(found, np.uint32),
                        probe_slot=np.array(slot, np.uint32))

    # --- pair / single front halves on the small index ---
    sets = {
        "pairs100": synth.simulate_pairs(tx, 3000, seed=31, read_len=100, sub_rate=0.005,
                                         indel_rate=0.0002),
        "pairs150div": synth.simulate_pairs(tx, 1500, seed=32, read_len=150, frag_mu=300,
                                            frag_sd=30, sub_rate=0.03, indel_rate=0.005,
                                            indel_len=(1, 8)),
        "pairs_mixed": synth.simulate_mixed_pairs(tx, 1500, seed=33),
        "pairs_long": synth.simulate_pairs(tx, 300, seed=34, read_len=260, frag_mu=400,
                                           frag_sd=30, sub_rate=0.02, indel_rate=0.002),
    }
    r1, r2 = synth.simulate_pairs(tx, 1000, seed=35, read_len=100, sub_rate=0.01)
    rr = np.random.default_rng(35)
    for rs in (r1, r2):
        rs.seq[rr.random(rs.seq.shape[0]) < 0.01] = ord("N")
    sets["pairs_n"] = (r1, r2)
    arrays = {}
    for name, (a, b) in sets.items():
        for wb in (1, 0):
            res = ref.align_pairs(a.copy(), b.copy(), wb)
            for k, v in records_to_arrays(res).items():
                arrays[f"{name}_wb{wb}_{k}"] = v
        for tag, rs in (("r1", a), ("r2", b)):
            arrays[f"{name}_{tag}_seq"] = rs.seq
            arrays[f"{name}_{tag}_off"] = rs.off
            arrays[f"{name}_{tag}_len"] = rs.len
    single = synth.simulate_single(tx, 2000, seed=36)
    for wb in (1, 0):
        res = ref.align_single(single.copy(), wb)
        for k, v in records_to_arrays(res).items():
            arrays[f"single_wb{wb}_{k}"] = v
    arrays["single_seq"], arrays["single_off"], arrays["single_len"] = single.seq, single.off, single.len
    np.savez_compressed(os.path.join(HERE, "candidates.npz"), **arrays)
    meta["pair_sets"] = sorted(sets)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print("golden vectors written:", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
