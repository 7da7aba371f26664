"""GPU parity: the CUDA path against the oracle, record for record."""
import numpy as np
import pytest

from hera_b200 import synth

pytestmark = pytest.mark.gpu


def _cmp(a, b):
    ca, cb = a.canonical(), b.canonical()
    bad = [i for i in range(len(ca)) if ca[i] != cb[i]]
    return bad, ca, cb


@pytest.mark.parametrize("write_bam", [1, 0])
def test_pairs_config1(config1, oracle1, gpu_ctx1, write_bam):
    _, tx, _ = config1
    r1, r2 = synth.simulate_pairs(tx, 20000, seed=7, read_len=100)
    g = gpu_ctx1.align_pairs(r1, r2, write_bam)
    o = oracle1.align_pairs(r1.copy(), r2.copy(), write_bam)
    bad, cg, co = _cmp(g, o)
    assert not bad, f"{len(bad)} mismatches, first {bad[0]}: gpu {cg[bad[0]]} oracle {co[bad[0]]}"
