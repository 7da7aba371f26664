"""The C-ABI library loads and exports every entry point include/hera_gpu.h
declares.  No compute calls (no GPU needed)."""
import ctypes as C
import os
import re

import pytest

from hera_b200 import api, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    txt = open(os.path.join(ROOT, "include", "hera_gpu.h")).read()
    return sorted(set(re.findall(r"^(?:int|void|const char) \*?\s*(hera_gpu_\w+)\s*\(", txt, re.M)))


def test_header_declares_entry_points():
    names = declared()
    for must in ("hera_gpu_ctx_create", "hera_gpu_align_pairs", "hera_gpu_align_pairs_flat",
                 "hera_gpu_align_single", "hera_gpu_align_pairs_device", "hera_gpu_ctx_destroy"):
        assert must in names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(build.LIB):
        pytest.skip("libhera_b200.so not built")
    lib = C.CDLL(build.LIB)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    lib.hera_gpu_abi_version.restype = C.c_int
    assert lib.hera_gpu_abi_version() == 2


def test_no_device_fails_loudly():
    """Without a CUDA device, context creation reports ENODEV instead of
    falling back to the CPU."""
    import torch
    if torch.cuda.is_available() or not os.path.exists(build.LIB):
        pytest.skip("a device is present / library not built")
    from hera_b200 import synth, index
    ann = synth.make_annotation(seed=7, genome_len=100_000, n_genes=5, n_transcripts=8)
    ix = index.build_index(synth.transcriptome(ann))
    with pytest.raises(api.HeraGpuError) as e:
        api.Context(ix)
    assert e.value.code == -1
