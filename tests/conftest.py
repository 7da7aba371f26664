"""Shared fixtures.  `-m gpu` tests need a CUDA device and the in-tree
libhera_b200.so; everything else runs on CPU.  The oracle (oracle/_ref,
built by `make -C oracle`) is the checker for both."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libhera_b200.so")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def config1():
    """Config-1 shaped data: 2 Mbp genome, 200 genes, 500 isoforms."""
    from hera_b200 import synth, index
    ann = synth.make_annotation(seed=1, genome_len=2_000_000, n_genes=200, n_transcripts=500)
    tx = synth.transcriptome(ann)
    ix = index.build_index(tx)
    return ann, tx, ix


@pytest.fixture(scope="session")
def config2s():
    """Config 2's gene and read model on a 40 Mbp genome: 6k genes, 20k
    transcripts, isoform families as in config 2 (the benched model at a
    size the oracle finishes in seconds)."""
    from hera_b200 import workloads
    return workloads.build("config2s", device="cuda" if gpu_available() else None)


@pytest.fixture(scope="session")
def family():
    """Paralog families larger than the per-read list capacities: 96
    transcripts sharing 600 bp (a read from it has 96 hits a strand and, at
    seed spacing 14, over 256 anchors), 40 sharing 400 bp, 30 unrelated."""
    from hera_b200 import index, synth
    tx = synth.family_transcriptome(21, families=((96, 600), (40, 400)), n_other=30)
    return tx, index.build_index(tx)


@pytest.fixture(scope="session")
def oracle1(config1):
    import oracle
    if not os.path.exists(oracle.ORACLE_SO):
        pytest.skip("oracle not built (make -C oracle)")
    return oracle.Oracle(config1[2])


@pytest.fixture(scope="session", params=["batched", "plain"])
def gpu_ctx1(request, config1):
    """A device context over the config-1 index, for each execution form."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    from hera_b200 import api
    ctx = api.Context(config1[2], max_batch=1 << 16, path=request.param)
    yield ctx
    ctx.close()
