"""The batched form's gap DP (sw_align_bits, hera_b200/csrc/hera_device.cuh)
compiled for the host and called the way k_dp_reg calls it: against the
reference's own SW_align outputs for the golden calls (tests/golden/
sw_align.npz) in both modes, and, in the score-only mode, its row-summary
form against the same DP keeping whole rows on random calls.  The GPU
suite runs the same golden calls through the kernels themselves
(test_gpu_units.py::test_gap_dp_golden)."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
CIGAR_CHARS = "MIDNSHP=XB"


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    so = str(tmp_path_factory.mktemp("dp") / "dp_host_check.so")
    subprocess.run([gxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-w", os.path.join(HERE, "dp_host_check.cpp"),
                    "-o", so], check=True)
    lib = C.CDLL(so)
    lib.dp_bits.restype = C.c_int
    lib.dp_bits.argtypes = [C.c_char_p, C.c_int, C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int),
                            C.c_void_p, C.POINTER(C.c_int), C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.dp_summaries_vs_rows.restype = C.c_long
    lib.dp_summaries_vs_rows.argtypes = [C.c_int, C.c_uint, C.POINTER(C.c_long), C.POINTER(C.c_long)]
    return lib


def _strs(buf, off):
    return [bytes(buf[off[i]:off[i + 1]]) for i in range(len(off) - 1)]


@pytest.mark.parametrize("wb", [1, 0])
def test_gap_dp_host_build_golden(lib, wb):
    """Every golden call the register form serves (the others are
    k_dp_generic's): score, CIGAR and mismatch bases equal the reference's."""
    d = np.load(os.path.join(GOLD, "sw_align.npz"))
    refs, qs = _strs(d["ref"], d["ref_off"]), _strs(d["q"], d["q_off"])
    cig = _strs(d[f"cigar_wb{wb}"], d[f"cigar_off_wb{wb}"])
    miss = _strs(d[f"miss_wb{wb}"], d[f"miss_off_wb{wb}"])
    ops = np.zeros(256, np.uint32)
    mb = np.zeros(256, np.uint8)
    score, n_ops, n_miss, flags = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    done, bad = 0, []
    for i, (r, q) in enumerate(zip(refs, qs)):
        e = int(d["err"][i])
        if not lib.dp_bits(r, len(r), q, len(q), e, wb, C.byref(score), ops.ctypes.data, C.byref(n_ops),
                           mb.ctypes.data, C.byref(n_miss), C.byref(flags)):
            continue
        done += 1
        got = (score.value, "".join(f"{int(x) >> 4}{CIGAR_CHARS[int(x) & 15]}" for x in ops[:n_ops.value]),
               bytes(mb[:n_miss.value]), flags.value)
        if got != (int(d[f"score_wb{wb}"][i]), cig[i].decode(), miss[i], 0):
            bad.append(i)
    assert done > 2500
    assert not bad, f"{len(bad)} of {done} golden calls differ, first {bad[:5]}"


def test_row_summaries_equal_whole_rows(lib):
    """The score-only mode's 2-byte row summaries give the whole-row DP's
    results, the shrink loop's path (soft clips) included."""
    n, clipped = C.c_long(), C.c_long()
    bad = lib.dp_summaries_vs_rows(60000, 11, C.byref(n), C.byref(clipped))
    assert bad == 0
    assert n.value > 50000 and clipped.value > n.value // 4
