"""Kernel-level GPU parity against the golden vectors the reference
produced: the mate-rescue DP (ssw_align, tests/golden/ssw_align.npz: score,
skip, CIGAR and miss chars) and the gap DP (SW_align,
tests/golden/sw_align.npz: score, CIGAR and miss chars in both WRITE_BAM
modes, through the batched form's own DP kernels)."""
import os
import re

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _strs(a, off):
    return [bytes(a[off[i]:off[i + 1]]) for i in range(len(off) - 1)]


def test_rescue_dp_golden():
    if not __import__("torch").cuda.is_available():
        pytest.skip("no CUDA device")
    from hera_b200 import api
    d = np.load(os.path.join(GOLD, "ssw_align.npz"))
    refs, reads = _strs(d["ref"], d["ref_off"]), _strs(d["read"], d["read_off"])
    cig, miss = _strs(d["cigar"], d["cigar_off"]), _strs(d["miss"], d["miss_off"])
    got, flags = api.unit_ssw(refs, reads)
    assert flags == 0, hex(flags)
    bad = [i for i, g in enumerate(got) if g != (int(d["score"][i]), int(d["skip"][i]), cig[i].decode(), miss[i])]
    assert not bad, (f"{len(bad)} of {len(got)} rescue DPs differ; first "
                     f"{[(i, got[i][:2], len(reads[i]), len(refs[i])) for i in bad[:5]]}")
    # the set holds CIGARs past the first pass's 96 ops (the wide form's cases)
    assert sum(1 for c in cig if len(re.findall(rb"[MIDNSX]", c)) > 96) >= 4

@pytest.mark.parametrize("wb", [1, 0])
def test_gap_dp_golden(wb):
    """All 3,000 reference SW_align calls: prefix (err < 0) and gap DPs at
    both error caps, empty queries, and windows shorter than error + 1 (the
    row-0 spill, computed by k_dp_generic)."""
    if not __import__("torch").cuda.is_available():
        pytest.skip("no CUDA device")
    from hera_b200 import api
    d = np.load(os.path.join(GOLD, "sw_align.npz"))
    refs, qs = _strs(d["ref"], d["ref_off"]), _strs(d["q"], d["q_off"])
    cig = _strs(d[f"cigar_wb{wb}"], d[f"cigar_off_wb{wb}"])
    miss = _strs(d[f"miss_wb{wb}"], d[f"miss_off_wb{wb}"])
    err = d["err"]
    rl = np.diff(d["ref_off"])
    spill = (rl < np.abs(err) + 2) & (np.diff(d["q_off"]) > 0)
    assert spill.sum() > 20   # the spill cases are in the set
    got, flags = api.unit_sw(refs, qs, err, wb)
    assert flags == 0, hex(flags)
    bad = [i for i in range(len(refs)) if got[i] != (int(d[f"score_wb{wb}"][i]), cig[i].decode(), miss[i])]
    assert not bad, (f"{len(bad)} of {len(refs)} SW_align vectors differ; first "
                     f"{[(i, got[i], int(d[f'score_wb{wb}'][i]), cig[i]) for i in bad[:3]]}")
