"""Class tables built by hand for the EM tests."""
import numpy as np

import oracle


def slow_table(n_trans: int) -> "oracle.ClassTable":
    """Triples of transcripts, each with one heavy shared class (1e5 reads)
    and a light class (1 read) on two of them, no single-transcript reads:
    on the config-1 index SQUAREM runs past its 50-round minimum here, so
    the convergence test decides when it stops."""
    lists, counts = [], []
    for i in range(0, n_trans - 2, 3):
        lists += [[i, i + 1, i + 2], [i, i + 1]]
        counts += [1e5, 1.0]
    ns = np.array([len(x) for x in lists], np.uint32)
    off = np.zeros(len(ns), np.uint64)
    off[1:] = np.cumsum(ns[:-1])
    return oracle.ClassTable(np.arange(len(ns), dtype=np.uint32), np.array(counts), ns, off,
                             np.concatenate([np.array(x, np.uint32) for x in lists]),
                             np.zeros(n_trans, np.uint32), 0, 0.0)
