#!/usr/bin/env python
"""Generate bam.npz in this directory from the reference program.

    make -C oracle && python tests/golden/make_bam_golden.py

The small seeded annotation of make_golden.py is indexed by the reference's
own tools (hera_build, which runs `hera index`), so GENE_MAP comes from the
reference.inf they write.  The reference's whole per-pair worker,
align_pair_read (src/hash_align.c:1717-1812), then runs with `-w`
(WRITE_BAM = 0) over the golden read sets of candidates.npz, and the
uncompressed BAM records it appends per pair (bam_write_pair,
src/bam_write.c:382-416) are stored with the gene map they were made with;
likewise align_single_read's records (bam_write_single, :418-446) for the
golden single reads.
"""
import ctypes as C
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hera_b200 import synth  # noqa: E402
import oracle  # noqa: E402
from make_golden import small_index  # noqa: E402

SETS = {"pairs100": 1200, "pairs150div": 600, "pairs_mixed": 600, "pairs_n": 600, "pairs_long": 300}


def main():
    ann, tx, ix = small_index()
    d = tempfile.mkdtemp()
    try:   # the reference's loader reads the index directory into memory
        synth.write_genome_fasta(ann, os.path.join(d, "g.fa"))
        synth.write_gtf(ann, os.path.join(d, "g.gtf"))
        shutil.copy(oracle.REF_HERA_BUILD, os.path.join(d, "hera_build"))
        shutil.copy(oracle.REFERENCE_BIN, os.path.join(d, "hera"))
        subprocess.run(["python3", os.path.join(d, "hera_build"), "--fasta", os.path.join(d, "g.fa"), "--gtf",
                        os.path.join(d, "g.gtf"), "--outdir", os.path.join(d, "idx")], check=True,
                       capture_output=True)
        gm = oracle.GeneMap(os.path.join(d, "idx", "reference.inf"), ix.n_trans)
        lib = C.CDLL(oracle.REFERENCE_SO)
        lib.refh_bam_setup(os.path.join(d, "idx").encode())
    finally:
        shutil.rmtree(d, ignore_errors=True)
    c = np.load(os.path.join(HERE, "candidates.npz"))
    out = {"gm_chr_len": gm.chr_len, "gm_exon_off": gm.exon_off, "gm_starts": gm.starts, "gm_ends": gm.ends,
           "gm_chr": gm.chr, "gm_gene": gm.gene}
    for name, n in SETS.items():
        r1 = synth.ReadSet(c[f"{name}_r1_seq"], c[f"{name}_r1_off"], c[f"{name}_r1_len"]).subset(np.arange(n))
        r2 = synth.ReadSet(c[f"{name}_r2_seq"], c[f"{name}_r2_off"], c[f"{name}_r2_len"]).subset(np.arange(n))
        q = [np.full(r1.seq.shape[0] + 1, ord("?"), np.uint8), np.full(r2.seq.shape[0] + 1, ord("?"), np.uint8)]
        nm = [oracle.read_names(n, 1), oracle.read_names(n, 2)]
        buf = np.zeros(1 << 26, np.uint8)
        off = np.zeros(n + 1, np.uint64)
        a1, a2 = r1.copy(), r2.copy()
        rc = lib.refh_bam_pairs(n, *oracle._bam_args(a1, a2, q, nm), C.c_void_p(buf.ctypes.data),
                                C.c_uint64(buf.size), C.c_void_p(off.ctypes.data))
        assert rc == 0
        out[f"{name}_bam"] = buf[:int(off[-1])].copy()
        out[f"{name}_bam_off"] = off
        out[f"{name}_n"] = np.array([n])
        print(name, n, "pairs,", int(off[-1]), "bytes of records")
    # single reads: align_single_read with `-w` (src/hash_align.c:1814-1853)
    n = 800
    rs = synth.ReadSet(c["single_seq"], c["single_off"], c["single_len"]).subset(np.arange(n))
    q = np.full(rs.seq.shape[0] + 1, ord("?"), np.uint8)
    nm = oracle.read_names(n, 1)
    buf = np.zeros(1 << 26, np.uint8)
    off = np.zeros(n + 1, np.uint64)
    a = rs.copy()
    rc = lib.refh_bam_single(n, C.c_void_p(a.seq.ctypes.data), C.c_void_p(a.off.ctypes.data),
                             C.c_void_p(a.len.ctypes.data), C.c_void_p(q.ctypes.data), C.c_void_p(nm.ctypes.data),
                             C.c_int32(nm.shape[1]), C.c_void_p(buf.ctypes.data), C.c_uint64(buf.size),
                             C.c_void_p(off.ctypes.data))
    assert rc == 0
    out["single_bam"], out["single_bam_off"], out["single_n"] = buf[:int(off[-1])].copy(), off, np.array([n])
    print("single", n, "reads,", int(off[-1]), "bytes of records")
    np.savez_compressed(os.path.join(HERE, "bam.npz"), **out)


if __name__ == "__main__":
    main()
