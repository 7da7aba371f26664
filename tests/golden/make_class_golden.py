#!/usr/bin/env python
"""Generate classes.npz in this directory from the reference program.

    make -C oracle && python tests/golden/make_class_golden.py

Expected values come from the reference's own code
(oracle/_ref/libhera_ref.so): its whole per-read worker, align_pair_read /
align_single_read (src/hash_align.c:1717-1853), run without `-w` over the
read sets stored in candidates.npz, after which the add_class state is read
back -- the class table in first-insertion order (XXH32 id, count,
transcript list), REF_INF->count, PAIRED and MEAN_FRAG's sum -- and the
reference's estimate_count (src/EM.c:315-387) over each of those tables
(em_val->grama and ->overlap, bit for bit).  Also XXH32 (src/xxhash.c) of
seeded random buffers of every length 0..96.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hera_b200 import synth  # noqa: E402
import oracle  # noqa: E402
from make_golden import small_index  # noqa: E402

SETS = ["pairs100", "pairs150div", "pairs_mixed", "pairs_long", "pairs_n"]


def main():
    ann, tx, ix = small_index()
    ref = oracle.Reference(ix)
    d = np.load(os.path.join(HERE, "candidates.npz"))
    out = {}
    rng = np.random.default_rng(77)
    bufs = [rng.integers(0, 256, n, dtype=np.uint8).tobytes() for n in range(97)]
    out["xxh_buf"] = np.frombuffer(b"".join(bufs), np.uint8)
    out["xxh_len"] = np.array([len(b) for b in bufs], np.int64)
    out["xxh_id"] = np.array([ref.xxh32(b) for b in bufs], np.uint32)
    for name in SETS + ["single"]:
        if name == "single":
            rs = synth.ReadSet(d["single_seq"].copy(), d["single_off"], d["single_len"])
            t = ref.classes(rs, None, ix.n_trans)
        else:
            r1 = synth.ReadSet(d[f"{name}_r1_seq"].copy(), d[f"{name}_r1_off"], d[f"{name}_r1_len"])
            r2 = synth.ReadSet(d[f"{name}_r2_seq"].copy(), d[f"{name}_r2_off"], d[f"{name}_r2_len"])
            t = ref.classes(r1, r2, ix.n_trans)
        out[f"{name}_ids"], out[f"{name}_counts"], out[f"{name}_ns"] = t.ids, t.counts, t.ns
        out[f"{name}_ref_off"], out[f"{name}_ref"], out[f"{name}_tx"] = t.ref_off, t.ref, t.tx_count
        out[f"{name}_paired"] = np.array([t.paired], np.uint32)
        out[f"{name}_mean_frag"] = np.array([t.mean_frag], np.float64)
        g, o = ref.em(t, ix.n_trans)
        out[f"{name}_em_grama"], out[f"{name}_em_overlap"] = g, o
        print(name, "classes", t.n_classes, "paired", t.paired, "one-transcript reads", int(t.tx_count.sum()))
    # a constructed table: triples of transcripts with one heavy shared
    # class and a light class on two of them, no single-transcript reads
    lists, counts = [], []
    for i in range(0, ix.n_trans - 2, 3):
        lists += [[i, i + 1, i + 2], [i, i + 1]]
        counts += [1e5, 1.0]
    ns = np.array([len(x) for x in lists], np.uint32)
    off = np.zeros(len(ns), np.uint64)
    off[1:] = np.cumsum(ns[:-1])
    slow = oracle.ClassTable(np.arange(len(ns), dtype=np.uint32), np.array(counts), ns, off,
                             np.concatenate([np.array(x, np.uint32) for x in lists]),
                             np.zeros(ix.n_trans, np.uint32), 0, 0.0)
    out["slow_counts"], out["slow_ns"], out["slow_ref_off"], out["slow_ref"] = slow.counts, ns, off, slow.ref
    out["slow_em_grama"], out["slow_em_overlap"] = ref.em(slow, ix.n_trans)
    np.savez_compressed(os.path.join(HERE, "classes.npz"), **out)


if __name__ == "__main__":
    main()
