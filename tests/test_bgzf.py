"""The BGZF encoder of the device path (hera_b200/csrc/hera_bgzf_core.h),
compiled for the host: every block a valid gzip member with the BGZF extra
field and a size within 64 KiB, and the whole decompressing to the input
(the bytes differ from zlib's, as any two DEFLATE encoders' do; a BAM
reader sees only the decompressed stream)."""
import ctypes as C
import gzip
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


@pytest.fixture(scope="module")
def enc(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    so = str(tmp_path_factory.mktemp("bgzf") / "bgzf_host_check.so")
    subprocess.run([gxx, "-O2", "-std=c++17", "-shared", "-fPIC", os.path.join(HERE, "bgzf_host_check.cpp"),
                    "-o", so], check=True)
    lib = C.CDLL(so)
    lib.bgzf_host.restype = C.c_longlong
    lib.bgzf_host.argtypes = [C.c_void_p, C.c_longlong, C.c_void_p, C.c_longlong]
    return lib


def _compress(lib, data: bytes) -> bytes:
    a = np.frombuffer(data, np.uint8).copy() if data else np.zeros(1, np.uint8)
    cap = len(data) + len(data) // 8 + 1024 * (len(data) // 0xff00 + 2)
    out = np.zeros(cap, np.uint8)
    n = lib.bgzf_host(a.ctypes.data, len(data), out.ctypes.data, cap)
    assert n >= 0
    return out[:n].tobytes()


def _blocks(z: bytes):
    o = 0
    while o < len(z):
        assert z[o:o + 4] == b"\x1f\x8b\x08\x04" and z[o + 12:o + 16] == b"BC\x02\x00"
        (bsize,) = struct.unpack_from("<H", z, o + 16)
        yield z[o:o + bsize + 1]
        o += bsize + 1
    assert o == len(z)


def _inputs():
    rng = np.random.default_rng(3)
    yield b""
    yield b"A"
    yield b"ACGT" * 5
    yield rng.integers(0, 256, 200_000, dtype=np.uint8).tobytes()          # incompressible: stored blocks
    yield (b"HTRAN0000000001" * 9000)[:0xff00]                             # one block exactly
    yield (b"HTRAN0000000001" * 9000)[:0xff00 + 1]                         # one byte over
    yield rng.integers(0, 4, 300_000, dtype=np.uint8).tobytes()            # small alphabet
    yield bytes(np.repeat(rng.integers(0, 256, 4000, dtype=np.uint8), rng.integers(1, 300, 4000)))   # runs
    d = np.load(os.path.join(GOLD, "bam.npz"))
    yield d["pairs100_bam"].tobytes()                                      # the reference's own BAM records


def test_bgzf_decompresses_to_input(enc):
    for data in _inputs():
        z = _compress(enc, data)
        blocks = list(_blocks(z))
        assert len(blocks) == max(1, -(-len(data) // 0xff00)) if data else len(blocks) == 0
        for blk in blocks:
            assert len(blk) <= 65536
            (isize,) = struct.unpack_from("<I", blk, len(blk) - 4)
            assert len(gzip.decompress(blk)) == isize
        assert gzip.decompress(z) == data if data else z == b""


def test_bgzf_compresses_bam_records(enc):
    d = np.load(os.path.join(GOLD, "bam.npz"))
    data = b"".join(d[f"{k}_bam"].tobytes() for k in ("pairs100", "pairs150div", "pairs_mixed", "pairs_n"))
    z = _compress(enc, data)
    assert gzip.decompress(z) == data
    assert len(z) < len(data) / 2
