"""The oracle restatement (oracle/hera_oracle.c) against golden vectors that
the reference program produced (tests/golden/make_golden.py).  CPU only."""
import json
import os

import numpy as np
import pytest

import oracle
from hera_b200 import index, synth

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _strs(buf, off):
    return [bytes(buf[off[i]:off[i + 1]]) for i in range(len(off) - 1)]


@pytest.fixture(scope="module")
def small():
    meta = json.load(open(os.path.join(GOLD, "golden.json")))
    p = dict(meta["index"])
    for k in ("exons", "intron"):
        p[k] = tuple(p[k])
    ann = synth.make_annotation(**p)
    tx = synth.transcriptome(ann)
    ix = index.build_index(tx)
    return meta, ix


@pytest.fixture(scope="module")
def orc(small):
    if not os.path.exists(oracle.ORACLE_SO):
        pytest.skip("oracle not built (make -C oracle)")
    return oracle.Oracle(small[1])


def test_generator_reproduces_index(small):
    from tests.golden.make_golden import index_digest
    meta, ix = small
    assert index_digest(ix) == meta["index_digest"]


@pytest.mark.parametrize("wb", [1, 0])
def test_sw_align_golden(orc, wb):
    d = np.load(os.path.join(GOLD, "sw_align.npz"))
    refs, qs = _strs(d["ref"], d["ref_off"]), _strs(d["q"], d["q_off"])
    cig = _strs(d[f"cigar_wb{wb}"], d[f"cigar_off_wb{wb}"])
    miss = _strs(d[f"miss_wb{wb}"], d[f"miss_off_wb{wb}"])
    bad = []
    for i, (r, q) in enumerate(zip(refs, qs)):
        got = orc.sw_align(r + b"\0" * 16, 0, q, len(r), len(q), int(d["err"][i]), wb)
        if got != (int(d[f"score_wb{wb}"][i]), cig[i].decode(), miss[i]):
            bad.append(i)
    assert not bad, f"{len(bad)} SW_align vectors differ, first {bad[0]}"


def test_ssw_align_golden(orc):
    d = np.load(os.path.join(GOLD, "ssw_align.npz"))
    refs, reads = _strs(d["ref"], d["ref_off"]), _strs(d["read"], d["read_off"])
    cig, miss = _strs(d["cigar"], d["cigar_off"]), _strs(d["miss"], d["miss_off"])
    bad = []
    for i, (r, q) in enumerate(zip(refs, reads)):
        got = orc.ssw_align(r, q)
        if got != (int(d["score"][i]), int(d["skip"][i]), cig[i].decode(), miss[i]):
            bad.append(i)
    assert not bad, f"{len(bad)} ssw_align vectors differ, first {bad[0]}"


def test_ssw_saturation_cases_present():
    """The golden set holds reads > 252 bp whose u8 cells saturate."""
    d = np.load(os.path.join(GOLD, "ssw_align.npz"))
    lens = np.diff(d["read_off"])
    assert (lens > 252).sum() > 20


def test_kmer_ids_and_probes_golden(orc, small):
    import ctypes as C
    d = np.load(os.path.join(GOLD, "kmers.npz"))
    kms = d["kmer"].reshape(-1, 31)
    for k, want in zip(kms, d["ids"]):
        assert orc.get_index(k.tobytes(), 0) == int(want)
    orc.lib.ho_hash_get.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(C.c_uint32)]
    for pid, f, s in zip(d["probe_ids"], d["probe_found"], d["probe_slot"]):
        found = C.c_uint32(0)
        slot = orc.lib.ho_hash_get(C.addressof(orc.cix), int(pid), C.byref(found))
        assert found.value == int(f)
        if f:
            assert slot == int(s)


def _golden_result(d, key):
    res = oracle.Result(d[f"{key}_recs"].shape[0], 1, 1, 1)
    res.recs = d[f"{key}_recs"]
    res.pos_pool, res.p_pool = d[f"{key}_pos"], d[f"{key}_p"]
    res.op_pool, res.miss_pool = d[f"{key}_ops"], d[f"{key}_miss"]
    return res.canonical()


SETS = ["pairs100", "pairs150div", "pairs_mixed", "pairs_long", "pairs_n"]


@pytest.mark.parametrize("name", SETS)
@pytest.mark.parametrize("wb", [1, 0])
def test_pair_records_golden(orc, name, wb):
    d = np.load(os.path.join(GOLD, "candidates.npz"))
    r1 = synth.ReadSet(d[f"{name}_r1_seq"].copy(), d[f"{name}_r1_off"], d[f"{name}_r1_len"])
    r2 = synth.ReadSet(d[f"{name}_r2_seq"].copy(), d[f"{name}_r2_off"], d[f"{name}_r2_len"])
    got = orc.align_pairs(r1, r2, wb).canonical()
    want = _golden_result(d, f"{name}_wb{wb}")
    bad = [i for i in range(len(want)) if got[i] != want[i]]
    assert not bad, f"{name}: {len(bad)} records differ, first {bad[0]}: {got[bad[0]]} vs {want[bad[0]]}"


@pytest.mark.parametrize("wb", [1, 0])
def test_single_records_golden(orc, wb):
    d = np.load(os.path.join(GOLD, "candidates.npz"))
    rs = synth.ReadSet(d["single_seq"].copy(), d["single_off"], d["single_len"])
    got = orc.align_single(rs, wb).canonical()
    want = _golden_result(d, f"single_wb{wb}")
    assert got == want


def test_xxh32_golden(orc):
    """XXH32 as add_class keys classes with it (src/hash_align.c:1576)."""
    d = np.load(os.path.join(GOLD, "classes.npz"))
    buf, lens = d["xxh_buf"].tobytes(), d["xxh_len"]
    off = np.concatenate([[0], np.cumsum(lens)])
    for k in range(len(lens)):
        assert orc.xxh32(buf[off[k]:off[k + 1]]) == int(d["xxh_id"][k]), f"length {lens[k]}"


def _golden_classes(d, name):
    return oracle.ClassTable(d[f"{name}_ids"], d[f"{name}_counts"], d[f"{name}_ns"], d[f"{name}_ref_off"],
                             d[f"{name}_ref"], d[f"{name}_tx"], int(d[f"{name}_paired"][0]),
                             float(d[f"{name}_mean_frag"][0]))


def _golden_records(d, key):
    res = oracle.Result(d[f"{key}_recs"].shape[0], 1, 1, 1)
    res.recs = d[f"{key}_recs"]
    res.pos_pool, res.p_pool = d[f"{key}_pos"], d[f"{key}_p"]
    return res


@pytest.mark.parametrize("name", SETS + ["single"])
def test_classes_golden(orc, name):
    """The host tail's add_class calls restated over the golden records give
    the class table, REF_INF->count, PAIRED and MEAN_FRAG that the
    reference's own worker built from the same reads."""
    c = np.load(os.path.join(GOLD, "candidates.npz"))
    d = np.load(os.path.join(GOLD, "classes.npz"))
    got = orc.classes([_golden_records(c, f"{name}_wb1")], paired=name != "single")
    want = _golden_classes(d, name)
    assert got.key() == want.key()


def _slow_table(d, n_trans):
    return oracle.ClassTable(np.arange(len(d["slow_ns"]), dtype=np.uint32), d["slow_counts"], d["slow_ns"],
                             d["slow_ref_off"], d["slow_ref"], np.zeros(n_trans, np.uint32), 0, 0.0)


@pytest.mark.parametrize("name", SETS + ["single", "slow"])
def test_em_golden(orc, small, name):
    """estimate_count restated, over the golden class tables, against the
    reference's own EM on the same tables: bit for bit."""
    d = np.load(os.path.join(GOLD, "classes.npz"))
    t = _slow_table(d, small[1].n_trans) if name == "slow" else _golden_classes(d, name)
    g, o, rounds = orc.em(t)
    assert np.array_equal(g.view(np.uint64), d[f"{name}_em_grama"].view(np.uint64))
    assert np.array_equal(o.view(np.uint64), d[f"{name}_em_overlap"].view(np.uint64))
