"""The combining of concurrent drop-in calls (hera_b200/csrc/hera_combine.h),
compiled for the host and driven by threads with a fake batch function:
every request runs in exactly one batch and gets its own result, one batch
runs at a time, a batch holds one kind of request within the pair budget,
and concurrent callers do share batches."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    so = str(tmp_path_factory.mktemp("comb") / "combine_check.so")
    subprocess.run([gxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-pthread", os.path.join(HERE, "combine_check.cpp"),
                    "-o", so], check=True)
    lib = C.CDLL(so)
    lib.combine_check.restype = C.c_int
    lib.combine_check.argtypes = [C.c_int, C.c_int, C.c_int64, C.c_int, C.c_uint, C.POINTER(C.c_ulonglong),
                                  C.POINTER(C.c_ulonglong)]
    return lib


@pytest.mark.parametrize("threads,kinds,budget", [(1, 1, 10_000), (16, 1, 1 << 40), (16, 2, 20_000), (8, 3, 1)])
def test_every_request_runs_once_in_a_valid_batch(lib, threads, kinds, budget):
    calls = 200
    nb, mx = C.c_ulonglong(), C.c_ulonglong()
    bad = lib.combine_check(threads, calls, budget, kinds, 5, C.byref(nb), C.byref(mx))
    assert bad == 0
    assert 1 <= nb.value <= threads * calls
    if threads == 1 or budget == 1:
        assert mx.value == 1 and nb.value == threads * calls   # nothing to share
    else:
        assert mx.value > 1 and nb.value < threads * calls      # concurrent calls shared batches
