"""Live cross-check of the oracle against the reference program built here
(oracle/_ref/libhera_ref.so); skipped where the reference was not built."""
import numpy as np
import pytest

import oracle
from tests import em_cases
from hera_b200 import synth, workloads

pytestmark = pytest.mark.skipif(not oracle.reference_available(), reason="reference not built")


@pytest.fixture(scope="module")
def both(config1):
    ann, tx, ix = config1
    return ann, tx, oracle.Oracle(ix), oracle.Reference(ix)


@pytest.mark.parametrize("wl", ["config1", "config3", "config4"])
def test_pairs_match_reference(both, wl):
    ann, tx, o, ref = both
    r1, r2 = workloads.pairs(wl, ann, tx, 3000, seed=101)
    for wb in (1, 0):
        a = o.align_pairs(r1.copy(), r2.copy(), wb).canonical()
        b = ref.align_pairs(r1.copy(), r2.copy(), wb).canonical()
        assert a == b


def test_reads_modified_like_reference(both):
    """Lower-case a/c/g/t come back upper-case from the front half."""
    ann, tx, o, ref = both
    r1, r2 = synth.simulate_pairs(tx, 500, seed=102)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    r1.seq[:] = np.where(np.isin(r1.seq, acgt), r1.seq + 32, r1.seq)
    a1, a2, b1, b2 = r1.copy(), r2.copy(), r1.copy(), r2.copy()
    o.align_pairs(a1, a2, 1)
    ref.align_pairs(b1, b2, 1)
    assert np.array_equal(a1.seq, b1.seq) and np.array_equal(a2.seq, b2.seq)
    assert not np.isin(a1.seq, np.frombuffer(b"acgt", np.uint8)).any()


@pytest.mark.parametrize("wl", ["config1", "config4"])
def test_classes_match_reference(both, wl):
    """add_class restated over the oracle's records, in batches, against the
    reference's whole worker (align_pair_read, add_class included)."""
    ann, tx, o, ref = both
    r1, r2 = workloads.pairs(wl, ann, tx, 6000, seed=103)
    want = ref.classes(r1, r2, o.ix.n_trans)
    whole = o.align_pairs(r1.copy(), r2.copy(), 1)
    assert o.classes([whole]).key() == want.key()
    parts = [o.align_pairs(r1.subset(np.arange(a, b)), r2.subset(np.arange(a, b)), 1) for a, b in ((0, 1000), (1000, 3500), (3500, 6000))]
    assert o.classes(parts).key() == want.key()


def test_single_classes_match_reference(both):
    ann, tx, o, ref = both
    rs = synth.simulate_single(tx, 3000, seed=104)
    want = ref.classes(rs, None, o.ix.n_trans)
    assert o.classes([o.align_single(rs.copy(), 1)], paired=False).key() == want.key()


@pytest.mark.parametrize("wl", ["config1", "config3", "config4"])
def test_em_matches_reference(both, wl):
    """estimate_count restated == the reference's, bit for bit, on the class
    table of 8,000 pairs."""
    ann, tx, o, ref = both
    r1, r2 = workloads.pairs(wl, ann, tx, 8000, seed=105)
    t = o.classes([o.align_pairs(r1.copy(), r2.copy(), 1)])
    g, ov, _ = o.em(t)
    G, OV = ref.em(t, o.ix.n_trans)
    assert np.array_equal(g.view(np.uint64), G.view(np.uint64))
    assert np.array_equal(ov.view(np.uint64), OV.view(np.uint64))


def test_em_past_minimum_rounds_matches_reference(both):
    ann, tx, o, ref = both
    t = em_cases.slow_table(o.ix.n_trans)
    g, ov, rounds = o.em(t)
    assert rounds > 50
    G, OV = ref.em(t, o.ix.n_trans)
    assert np.array_equal(g.view(np.uint64), G.view(np.uint64))
    assert np.array_equal(ov.view(np.uint64), OV.view(np.uint64))


def test_config2s_pairs_match_reference(config2s):
    """The oracle against the reference on config 2's isoform structure
    (6k genes, 20k transcripts), both WRITE_BAM modes."""
    ann, tx, ix = config2s
    o, ref = oracle.Oracle(ix), oracle.Reference(ix)
    r1, r2 = workloads.pairs("config2s", ann, tx, 10000, seed=106)
    for wb in (1, 0):
        assert o.align_pairs(r1.copy(), r2.copy(), wb).canonical() == \
            ref.align_pairs(r1.copy(), r2.copy(), wb).canonical()


@pytest.mark.parametrize("mate2_random", [False, True])
def test_long_lists_match_reference(family, mate2_random):
    """Reads with 96 hits a strand (over 256 anchors at spacing 14), and
    mates that need a rescue over every family member: the oracle's lists
    are unbounded like the reference's."""
    tx, ix = family
    o, ref = oracle.Oracle(ix), oracle.Reference(ix)
    r1, r2 = synth.family_pairs(tx, 400, seed=107, shared=600, mate2_random=mate2_random)
    for wb in (1, 0):
        a = o.align_pairs(r1.copy(), r2.copy(), wb)
        assert a.canonical() == ref.align_pairs(r1.copy(), r2.copy(), wb).canonical()
    assert int(a.recs["n"].max()) > 64
