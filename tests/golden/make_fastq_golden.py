#!/usr/bin/env python
"""Generate tests/golden/fastq.npz from the reference program.

    make -C oracle && python tests/golden/make_fastq_golden.py

Every expected value comes from the reference's own FASTQ reader
(get_read_from_fq_buffer, src/read.c:11-63, in oracle/_ref/libhera_ref.so)
driven by the read loops of align_pool_pair / align_pool_single
(src/hash_align.c:1878-1929, 1966-1998).  The inputs are the seeded chunk
buffers of tests/fastq_cases.py (well-formed and malformed).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
import fastq_cases  # noqa: E402

PAIR_SEED, PAIR_COUNT = 21, 150
SINGLE_SEED, SINGLE_COUNT = 22, 80


def _pack(bufs):
    off = np.zeros(len(bufs) + 1, np.int64)
    off[1:] = np.cumsum([len(b) for b in bufs])
    return np.frombuffer(b"".join(bufs), np.uint8), off


def main():
    pairs = fastq_cases.pair_cases(PAIR_SEED, PAIR_COUNT, max_n=10, max_len=160)
    singles = fastq_cases.single_cases(SINGLE_SEED, SINGLE_COUNT, max_n=10, max_len=160)
    out = {}
    for tag, cases in (("pair", pairs), ("single", singles)):
        res, recs = [], []
        for c in cases:
            r = oracle.ref_parse_fq_pairs(*c) if tag == "pair" else oracle.ref_parse_fq_single(c)
            res.append((r[0], r[2], r[3], r[4]))
            recs.append(r[1])
        if tag == "pair":
            out["pair_left"], out["pair_left_off"] = _pack([c[0] for c in cases])
            out["pair_right"], out["pair_right_off"] = _pack([c[1] for c in cases])
        else:
            out["single_buf"], out["single_off"] = _pack(cases)
        out[f"{tag}_result"] = np.array(res, np.int64)   # status, n, bad_file, bad_rec
        ro = np.zeros(len(recs) + 1, np.int64)
        ro[1:] = np.cumsum([len(r) for r in recs])
        out[f"{tag}_recs"] = np.concatenate(recs) if recs else np.zeros(0, oracle.FQ_DTYPE)
        out[f"{tag}_recs_off"] = ro
    np.savez_compressed(os.path.join(HERE, "fastq.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
