"""Python mirror of the C ABI in include/hera_gpu.h (ctypes).

``Context`` owns one device copy of a hera index and runs the hot path:
``align_pairs`` is the batched replacement of the per-pair
check_in_transcriptome + intersect2 front half of hera's align_pair_read
(src/hash_align.c:1724-1733), ``align_single`` of align_single_read's two
get_position calls (src/hash_align.c:1822-1823).  Results come back as
``Result`` objects holding the flat hera_cand_rec records.

The library is hera_b200/libhera_b200.so, built in-tree by hera_b200.build.
There is no CPU fallback: a missing library or device raises.
"""
from __future__ import annotations

import ctypes as C
import time
import os
from typing import List, Optional

import numpy as np

from . import build as _build

LIB_PATH = _build.LIB

HERA_GPU_OK = 0
ERRORS = {-1: "ENODEV", -2: "ECUDA", -3: "ENOMEM", -4: "EINVAL", -5: "ECAPACITY", -6: "ETIMEOUT",
          -7: "EFORMAT", -8: "ECANCELED"}
HERA_GPU_ECAPACITY = -5
HERA_GPU_EFORMAT = -7
HERA_GPU_ECANCELED = -8
MAX_READ = 320
CIGAR_CHARS = "MIDNSHP=XB"

REC_DTYPE = np.dtype([
    ("n", "<i4", (2,)), ("err", "<i4", (2,)), ("pair", "<i4"),
    ("list_off", "<u4", (2,)), ("cig_off", "<u4", (2,)), ("miss_off", "<u4", (2,)),
    ("n_cigar", "<u2", (2,)), ("n_miss", "<u2", (2,)),
])


class HeraGpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"hera_gpu {ERRORS.get(code, code)}: {msg}")
        self.code = code


class FastqFormatError(HeraGpuError):
    """A chunk hera's reader rejects ("Wrong format of file"): file 1 or 2
    of a pair (1 for single reads) and the 0-based read of that file."""

    def __init__(self, code: int, msg: str, bad_file: int, bad_read: int):
        super().__init__(code, f"{msg} (file {bad_file}, read {bad_read})")
        self.bad_file = bad_file
        self.bad_read = bad_read


# one read of a FASTQ chunk (hera_gpu_fastq_rec): byte offsets into its buffer
FQ_DTYPE = np.dtype([("name", "<i8"), ("seq", "<i8"), ("qual", "<i8"),
                     ("name_len", "<i4"), ("len", "<i4")])


class FastqStats(C.Structure):
    _fields_ = [("h2d_ms", C.c_float), ("parse_ms", C.c_float), ("gather_ms", C.c_float),
                ("launches", C.c_int32), ("bytes", C.c_int64), ("reads", C.c_int64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class _IndexView(C.Structure):
    _fields_ = [("n_trans", C.c_uint32), ("len", C.c_void_p), ("find", C.c_void_p),
                ("seq", C.c_void_p), ("bucket_n", C.c_void_p), ("buckets", C.c_void_p),
                ("n_buckets", C.c_uint64), ("pos", C.c_void_p), ("p", C.c_void_p),
                ("n_pos", C.c_uint32)]


class _Options(C.Structure):
    _fields_ = [("device", C.c_int), ("max_batch", C.c_uint32), ("scratch_bytes", C.c_uint64),
                ("path", C.c_int), ("lanes", C.c_int)]


PATH_BATCHED = 0
PATH_PLAIN = 1


class _Result(C.Structure):
    _fields_ = [("recs", C.c_void_p), ("pos_pool", C.c_void_p), ("p_pool", C.c_void_p),
                ("op_pool", C.c_void_p), ("miss_pool", C.c_void_p),
                ("list_cap", C.c_uint64), ("op_cap", C.c_uint64), ("miss_cap", C.c_uint64),
                ("list_used", C.c_uint64), ("op_used", C.c_uint64), ("miss_used", C.c_uint64)]


class _Reads(C.Structure):
    _fields_ = [("seq", C.c_void_p), ("off", C.c_void_p), ("len", C.c_void_p)]


class Tuning(C.Structure):
    _fields_ = [("build_blocks_per_sm", C.c_int), ("rescue_warps_per_block", C.c_int), ("state", C.c_int),
                ("n_build", C.c_int), ("n_rescue", C.c_int), ("build_cand", C.c_int * 8),
                ("build_ms", C.c_float * 8), ("rescue_cand", C.c_int * 4), ("rescue_ms", C.c_float * 4)]

    def as_dict(self) -> dict:
        return {"build_blocks_per_sm": self.build_blocks_per_sm,
                "rescue_warps_per_block": self.rescue_warps_per_block,
                "state": ("defaults", "autotuned", "pinned")[self.state],
                "build_trials_ms": {int(self.build_cand[i]): round(float(self.build_ms[i]), 4)
                                    for i in range(self.n_build)},
                "rescue_trials_ms": {int(self.rescue_cand[i]): round(float(self.rescue_ms[i]), 4)
                                     for i in range(self.n_rescue)}}


class _ServerOptions(C.Structure):
    _fields_ = [("batch_pairs", C.c_uint32), ("max_slots", C.c_int), ("hbm_reserve", C.c_uint64),
                ("write_bam", C.c_int), ("max_samples", C.c_uint32), ("borrow_reads", C.c_int)]


class ChunkInfo(C.Structure):
    _fields_ = [("sample", C.c_uint32), ("n", C.c_int32), ("submit_ms", C.c_double),
                ("admit_ms", C.c_double), ("done_ms", C.c_double), ("batches", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class SampleStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("pairs", "mapped", "paired", "hits", "cigar_ops")] + [
        ("reserved", C.c_uint64 * 3)]

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_[:5]}


class ServerStats(C.Structure):
    _fields_ = [("slots", C.c_int), ("slot_bytes", C.c_uint64), ("chunks_done", C.c_uint64),
                ("pairs_done", C.c_uint64), ("batches", C.c_uint64), ("p50_ms", C.c_float),
                ("p99_ms", C.c_float), ("p50_wait_ms", C.c_float), ("p99_wait_ms", C.c_float),
                ("pairs_per_s", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Timing(C.Structure):
    _fields_ = [(k, C.c_float) for k in ("h2d_ms", "seed_ms", "position_ms", "resolve_ms",
                                         "rescue_ms", "pack_ms", "d2h_ms", "total_ms",
                                         "build_ms", "dp_ms")] + [
        ("launches", C.c_uint32), ("rescue_rounds", C.c_uint32), ("lookups", C.c_uint64),
        ("dp_jobs", C.c_uint64), ("dp_calls", C.c_uint64)] + [
        (k, C.c_float) for k in ("seed_kernel_ms", "dp_kernel_ms", "rescue_kernel_ms",
                                 "host_stage_ms", "host_out_ms")] + [
        (k, C.c_uint64) for k in ("probes", "seed_hits", "sw_cells", "ssw_cells", "wide_items")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


class _ClassTable(C.Structure):
    _fields_ = [("class_cap", C.c_uint32), ("id", C.c_void_p), ("count", C.c_void_p), ("n", C.c_void_p),
                ("list_off", C.c_void_p), ("list_cap", C.c_uint64), ("list", C.c_void_p),
                ("tx_count", C.c_void_p), ("n_classes", C.c_uint32), ("list_used", C.c_uint64),
                ("paired", C.c_uint32), ("mean_frag_sum", C.c_double)]


class _GeneMap(C.Structure):
    _fields_ = [("n_chr", C.c_uint32), ("chr_len", C.c_void_p), ("exon_off", C.c_void_p), ("starts", C.c_void_p),
                ("ends", C.c_void_p), ("chr", C.c_void_p), ("gene", C.c_void_p)]


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load libhera_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `python -m hera_b200.build`")
    lib = C.CDLL(path)
    lib.hera_gpu_abi_version.restype = C.c_int
    lib.hera_gpu_ctx_create.restype = C.c_int
    lib.hera_gpu_ctx_create.argtypes = [C.POINTER(_IndexView), C.POINTER(_Options), C.POINTER(C.c_void_p)]
    lib.hera_gpu_ctx_destroy.argtypes = [C.c_void_p]
    lib.hera_gpu_last_error.restype = C.c_char_p
    lib.hera_gpu_last_error.argtypes = [C.c_void_p]
    lib.hera_gpu_align_pairs_flat.argtypes = [C.c_void_p, C.POINTER(_Reads), C.POINTER(_Reads),
                                              C.c_int32, C.c_int, C.POINTER(_Result)]
    lib.hera_gpu_align_single_flat.argtypes = [C.c_void_p, C.POINTER(_Reads), C.c_int32, C.c_int,
                                               C.POINTER(_Result)]
    lib.hera_gpu_align_pairs_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_int32, C.c_int32, C.c_int, C.c_void_p]
    lib.hera_gpu_fetch_result.argtypes = [C.c_void_p, C.POINTER(_Result)]
    lib.hera_gpu_get_timing.argtypes = [C.c_void_p, C.POINTER(Timing)]
    lib.hera_gpu_stream.restype = C.c_void_p
    lib.hera_gpu_stream.argtypes = [C.c_void_p]
    lib.hera_gpu_dpx_peak.argtypes = [C.c_int, C.c_float, C.POINTER(C.c_double)]
    lib.hera_gpu_get_tuning.argtypes = [C.c_void_p, C.POINTER(Tuning)]
    lib.hera_gpu_host_register.argtypes = [C.c_void_p, C.c_size_t]
    lib.hera_gpu_unit_ssw.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_int32, C.POINTER(C.c_int32)]
    lib.hera_gpu_unit_sw.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_int32, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]
    lib.hera_gpu_host_unregister.argtypes = [C.c_void_p]
    lib.hera_gpu_server_create.argtypes = [C.c_void_p, C.POINTER(_ServerOptions), C.POINTER(C.c_void_p)]
    lib.hera_gpu_server_submit.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(_Reads), C.POINTER(_Reads),
                                           C.c_int32, C.POINTER(C.c_uint64)]
    lib.hera_gpu_server_wait.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(_Result), C.POINTER(ChunkInfo)]
    lib.hera_gpu_server_get_sample_stats.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(SampleStats)]
    lib.hera_gpu_server_get_stats.argtypes = [C.c_void_p, C.POINTER(ServerStats)]
    lib.hera_gpu_server_destroy.argtypes = [C.c_void_p]
    lib.hera_gpu_set_tuning.argtypes = [C.c_void_p, C.POINTER(Tuning)]
    lib.hera_gpu_parse_fastq_pairs.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                               C.c_void_p, C.c_int32, C.POINTER(C.c_int32),
                                               C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
    lib.hera_gpu_parse_fastq_single.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int32,
                                                C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
    lib.hera_gpu_align_fastq_pairs.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                               C.c_int, C.c_void_p, C.c_int32, C.POINTER(C.c_int32),
                                               C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(_Result)]
    lib.hera_gpu_get_fastq_stats.argtypes = [C.c_void_p, C.POINTER(FastqStats)]
    lib.hera_gpu_classes_create.argtypes = [C.c_void_p, C.c_uint32, C.c_uint64, C.POINTER(C.c_void_p)]
    lib.hera_gpu_classes_destroy.argtypes = [C.c_void_p]
    lib.hera_gpu_classes_add_last.argtypes = [C.c_void_p, C.c_void_p]
    lib.hera_gpu_classes_add_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                                C.c_int, C.c_void_p]
    lib.hera_gpu_classes_em.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32),
                                        C.POINTER(C.c_float)]
    lib.hera_gpu_bam_create.argtypes = [C.c_void_p, C.POINTER(_GeneMap), C.POINTER(C.c_void_p)]
    lib.hera_gpu_bam_destroy.argtypes = [C.c_void_p]
    lib.hera_gpu_bam_last_error.restype = C.c_char_p
    lib.hera_gpu_bam_last_error.argtypes = [C.c_void_p]
    lib.hera_gpu_bam_pairs.argtypes = [C.c_void_p, C.POINTER(_Result), C.c_int32, C.POINTER(_Reads), C.POINTER(_Reads),
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                       C.c_uint64, C.c_void_p, C.POINTER(C.c_float)]
    lib.hera_gpu_classes_load.argtypes = [C.c_void_p, C.POINTER(_ClassTable)]
    lib.hera_gpu_classes_add_host.argtypes = [C.c_void_p, C.POINTER(_Result), C.c_int32, C.c_int]
    lib.hera_gpu_classes_fetch.argtypes = [C.c_void_p, C.POINTER(_ClassTable)]
    lib.hera_gpu_classes_timing.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_uint32)]
    lib.hera_gpu_classes_last_error.restype = C.c_char_p
    lib.hera_gpu_classes_last_error.argtypes = [C.c_void_p]
    _lib = lib
    return lib


def dpx_peak(device: int = 0, ms: float = 50.0) -> float:
    """Thread-level __viaddmin_s16x2 instructions per second on `device`
    (each updates two 16-bit lanes): the measured DPX issue rate."""
    lib = load_library()
    out = C.c_double()
    rc = lib.hera_gpu_dpx_peak(device, ms, C.byref(out))
    if rc != HERA_GPU_OK:
        raise HeraGpuError(rc, "DPX probe failed")
    return out.value


def host_register(a: np.ndarray) -> None:
    """Page-lock a numpy array reused across calls (reads or result pools):
    calls then copy it to or from the device without the pinned staging."""
    lib = load_library()
    rc = lib.hera_gpu_host_register(C.c_void_p(a.ctypes.data), C.c_size_t(a.nbytes))
    if rc != HERA_GPU_OK:
        raise HeraGpuError(rc, "cudaHostRegister failed")


def host_unregister(a: np.ndarray) -> None:
    lib = load_library()
    lib.hera_gpu_host_unregister(C.c_void_p(a.ctypes.data))


def unit_ssw(refs, reads, device: int = 0, cap: int = 1344):
    """ssw_align as the mate-rescue kernel computes it (the wide pass's form
    for CIGARs past the first pass's capacities), for lists of ASCII
    (window, read) pairs: [(score, skip, cigar, miss)] (a kernel-level check
    against the reference's golden vectors)."""
    lib = load_library()
    n = len(refs)
    rcat = np.frombuffer(b"".join(refs), np.uint8).copy()
    qcat = np.frombuffer(b"".join(reads), np.uint8).copy()
    roff = np.zeros(n + 1, np.int64)
    roff[1:] = np.cumsum([len(r) for r in refs])
    qoff = np.zeros(n + 1, np.int64)
    qoff[1:] = np.cumsum([len(q) for q in reads])
    score, skip = np.zeros(n, np.int32), np.zeros(n, np.int32)
    ops = np.zeros(n * cap, np.uint32)
    miss = np.zeros(n * cap, np.uint8)
    n_ops, n_miss = np.zeros(n, np.int32), np.zeros(n, np.int32)
    flags = C.c_int32(0)
    rc = lib.hera_gpu_unit_ssw(device, _ptr(rcat), _ptr(roff), _ptr(qcat), _ptr(qoff), n, _ptr(score), _ptr(skip),
                               _ptr(ops), _ptr(n_ops), _ptr(miss), _ptr(n_miss), cap, C.byref(flags))
    if rc != HERA_GPU_OK:
        raise HeraGpuError(rc, "unit ssw failed")
    out = []
    for i in range(n):
        o = ops[i * cap:i * cap + min(int(n_ops[i]), cap)]
        cig = "".join(f"{int(x) >> 4}{CIGAR_CHARS[int(x) & 15]}" for x in o)
        out.append((int(score[i]), int(skip[i]), cig, bytes(miss[i * cap:i * cap + min(int(n_miss[i]), cap)])))
    return out, flags.value


def unit_sw(refs, qs, errs, write_bam: int, device: int = 0, cap: int = 64):
    """SW_align as the batched form's gap-DP kernels compute it, for lists
    of ASCII windows, queries and error caps: [(score, cigar, miss)] (a
    kernel-level check against the reference's golden vectors)."""
    lib = load_library()
    n = len(refs)
    rcat = np.frombuffer(b"".join(refs), np.uint8).copy()
    qcat = np.frombuffer(b"".join(qs), np.uint8).copy()
    roff = np.zeros(n + 1, np.int64)
    roff[1:] = np.cumsum([len(r) for r in refs])
    qoff = np.zeros(n + 1, np.int64)
    qoff[1:] = np.cumsum([len(q) for q in qs])
    err = np.asarray(errs, np.int32)
    score = np.zeros(n, np.int32)
    ops = np.zeros(n * cap, np.uint32)
    miss = np.zeros(n * cap, np.uint8)
    n_ops, n_miss = np.zeros(n, np.int32), np.zeros(n, np.int32)
    flags = C.c_int32(0)
    rc = lib.hera_gpu_unit_sw(device, _ptr(rcat), _ptr(roff), _ptr(qcat), _ptr(qoff), _ptr(err), n, write_bam,
                              _ptr(score), _ptr(ops), _ptr(n_ops), _ptr(miss), _ptr(n_miss), cap, C.byref(flags))
    if rc != HERA_GPU_OK:
        raise HeraGpuError(rc, "unit sw failed")
    out = []
    for i in range(n):
        o = ops[i * cap:i * cap + min(int(n_ops[i]), cap)]
        cig = "".join(f"{int(x) >> 4}{CIGAR_CHARS[int(x) & 15]}" for x in o)
        out.append((int(score[i]), cig, bytes(miss[i * cap:i * cap + min(int(n_miss[i]), cap)])))
    return out, flags.value


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class Result:
    """Flat Candidate records (hera_cand_rec) plus their pools."""

    def __init__(self, n_recs: int, list_cap: int, op_cap: int, miss_cap: int):
        self._rec_buf = np.empty(max(n_recs, 1), dtype=REC_DTYPE)
        self.recs = self._rec_buf[:n_recs]
        self._alloc(list_cap, op_cap, miss_cap)

    def _alloc(self, list_cap, op_cap, miss_cap):
        self.pos_pool = np.empty(max(list_cap, 1), np.uint32)
        self.p_pool = np.empty(max(list_cap, 1), np.int32)
        self.op_pool = np.empty(max(op_cap, 1), np.uint32)
        self.miss_pool = np.empty(max(miss_cap, 1), np.uint8)
        self._bind(list_cap, op_cap, miss_cap)

    def _bind(self, list_cap, op_cap, miss_cap):
        base = self.recs.ctypes.data if self.recs.shape[0] else 0
        self.c = _Result(base, _ptr(self.pos_pool), _ptr(self.p_pool), _ptr(self.op_pool),
                         _ptr(self.miss_pool), list_cap, op_cap, miss_cap, 0, 0, 0)

    def arrays(self):
        """The host arrays a call writes (records and pools)."""
        return [self._rec_buf, self.pos_pool, self.p_pool, self.op_pool, self.miss_pool]

    def reuse(self, n_recs: int) -> "Result":
        """Make room for n_recs records, keeping the pools' storage."""
        if self._rec_buf.shape[0] < n_recs:
            self._rec_buf = np.empty(n_recs, dtype=REC_DTYPE)
        self.recs = self._rec_buf[:n_recs]
        self._bind(self.pos_pool.shape[0], self.op_pool.shape[0], self.miss_pool.shape[0])
        return self

    def candidate(self, i: int):
        """(pair, ((n, err, pos, p, cigar, miss) for strand 0, 1))."""
        r = self.recs[i]
        out = []
        for s in range(2):
            n = int(r["n"][s])
            lo = int(r["list_off"][s])
            co, nc = int(r["cig_off"][s]), int(r["n_cigar"][s])
            mo, nm = int(r["miss_off"][s]), int(r["n_miss"][s])
            cig = "".join(f"{int(o) >> 4}{CIGAR_CHARS[int(o) & 15]}" for o in self.op_pool[co:co + nc])
            out.append((n, int(r["err"][s]), tuple(self.pos_pool[lo:lo + n].tolist()),
                        tuple(self.p_pool[lo:lo + n].tolist()), cig,
                        bytes(self.miss_pool[mo:mo + nm])))
        return (int(r["pair"]), tuple(out))

    def canonical(self, lo: int = 0, hi: Optional[int] = None) -> List[tuple]:
        hi = self.recs.shape[0] if hi is None else hi
        return [self.candidate(i) for i in range(lo, hi)]


class Context:
    """One hera index resident on one GPU."""

    def __init__(self, index, device: int = 0, max_batch: int = 0, scratch_bytes: int = 0,
                 path: str = "batched", lanes: int = 0):
        self.lib = load_library()
        self.index = index
        v = _IndexView()
        self._keep = [np.ascontiguousarray(index.length, np.uint32),
                      np.ascontiguousarray(index.find, np.uint32),
                      np.ascontiguousarray(index.seq, np.uint8),
                      np.ascontiguousarray(index.bucket_n, np.uint32),
                      np.ascontiguousarray(index.buckets),
                      np.ascontiguousarray(index.pos, np.uint32),
                      np.ascontiguousarray(index.p, np.uint32)]
        ln, fd, sq, bn, bk, pos, p = self._keep
        v.n_trans, v.len, v.find, v.seq = index.n_trans, _ptr(ln), _ptr(fd), _ptr(sq)
        v.bucket_n, v.buckets, v.n_buckets = _ptr(bn), _ptr(bk), bk.shape[0]
        v.pos, v.p, v.n_pos = _ptr(pos), _ptr(p), pos.shape[0]
        if path not in ("batched", "plain"):
            raise ValueError(f"unknown path {path!r}")
        self.path = path
        opt = _Options(device, max_batch, scratch_bytes, PATH_PLAIN if path == "plain" else PATH_BATCHED,
                       lanes)
        h = C.c_void_p()
        rc = self.lib.hera_gpu_ctx_create(C.byref(v), C.byref(opt), C.byref(h))
        if rc != HERA_GPU_OK:
            raise HeraGpuError(rc, "context creation failed")
        self.h = h
        self._inflight = {}   # asynchronous calls: ticket -> (reads structs, result)
        self._keep = None

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.hera_gpu_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        if rc != HERA_GPU_OK:
            raise HeraGpuError(rc, self.lib.hera_gpu_last_error(self.h).decode())

    @staticmethod
    def _reads(rs) -> _Reads:
        return _Reads(_ptr(rs.seq), _ptr(rs.off), _ptr(rs.len))

    def _run(self, fn, n_recs, total_len, args, out: Optional[Result] = None) -> Result:
        if out is not None:
            res = out.reuse(n_recs)
        else:
            res = Result(n_recs, n_recs * 4 + 1024, n_recs * 4 + 1024, total_len // 8 + 1024)
        rc = fn(*args, C.byref(res.c))
        if rc == -5 and (res.c.list_used > res.c.list_cap or res.c.op_used > res.c.op_cap
                         or res.c.miss_used > res.c.miss_cap):
            res._alloc(res.c.list_used + 1, res.c.op_used + 1, res.c.miss_used + 1)
            rc = fn(*args, C.byref(res.c))
        self._check(rc)
        return res

    def align_pairs(self, r1, r2, write_bam: int = 1, out: Optional[Result] = None) -> Result:
        """Paired reads (synth.ReadSet-like: seq, off, len) -> 2 records per
        pair.  `out`: a Result to reuse (its storage is overwritten)."""
        a, b = self._reads(r1), self._reads(r2)
        return self._run(self.lib.hera_gpu_align_pairs_flat, 2 * r1.n,
                         int(r1.len.sum()) + int(r2.len.sum()),
                         (self.h, C.byref(a), C.byref(b), r1.n, write_bam), out)

    def submit_pairs(self, r1, r2, write_bam: int, out: Result) -> int:
        """Start an asynchronous flat call (hera_gpu_align_pairs_submit);
        returns a ticket.  r1, r2 and out must stay alive and untouched
        until complete_pairs(ticket); out's pools must be large enough."""
        a, b = self._reads(r1), self._reads(r2)
        res = out.reuse(2 * r1.n)
        t = C.c_uint64()
        self.lib.hera_gpu_align_pairs_submit.argtypes = [C.c_void_p, C.POINTER(_Reads), C.POINTER(_Reads), C.c_int32,
                                                         C.c_int, C.POINTER(_Result), C.POINTER(C.c_uint64)]
        self.lib.hera_gpu_align_pairs_complete.argtypes = [C.c_void_p, C.c_uint64]
        self._check(self.lib.hera_gpu_align_pairs_submit(self.h, C.byref(a), C.byref(b), r1.n, write_bam,
                                                         C.byref(res.c), C.byref(t)))
        self._inflight[t.value] = (a, b, res)   # the structs the call reads
        return t.value

    def complete_pairs(self, ticket: int) -> Result:
        a, b, res = self._inflight.pop(ticket)
        self._check(self.lib.hera_gpu_align_pairs_complete(self.h, ticket))
        return res

    def align_single(self, rs, write_bam: int = 1, out: Optional[Result] = None) -> Result:
        a = self._reads(rs)
        return self._run(self.lib.hera_gpu_align_single_flat, rs.n, int(rs.len.sum()),
                         (self.h, C.byref(a), rs.n, write_bam), out)

    def align_pairs_device(self, d_seq: int, d_off: int, d_len: int, n: int, max_len: int,
                           write_bam: int = 1, stream: Optional[int] = None) -> None:
        """Device-resident batch: pointers into HBM (2n reads, mates
        interleaved).  Results stay on the device until fetch()."""
        self._check(self.lib.hera_gpu_align_pairs_device(self.h, d_seq, d_off, d_len, n, max_len,
                                                         write_bam, stream))

    # struct read_inf (src/read.h:16-21) as a numpy record: seq, name, qual
    # pointers and the length
    READ_INF = np.dtype([("seq", "<u8"), ("name", "<u8"), ("qual", "<u8"), ("len", "<i4"), ("pad", "<i4")])

    @classmethod
    def _read_infs(cls, rs):
        """read_inf entries over a NUL-separated copy of the reads (the
        copy is returned too: it must outlive the call)."""
        lens = rs.len.astype(np.int64)
        total = int(lens.sum())
        starts = np.cumsum(lens) - lens
        within = np.arange(total) - np.repeat(starts, lens)
        dst = np.zeros(rs.n, np.int64)
        dst[1:] = np.cumsum(lens[:-1] + 1)
        buf = np.zeros(total + rs.n + 1, np.uint8)
        buf[np.repeat(dst, lens) + within] = rs.seq[np.repeat(rs.off, lens) + within]
        ri = np.zeros(rs.n, cls.READ_INF)
        ri["seq"] = buf.ctypes.data + dst
        ri["len"] = rs.len
        return ri, buf

    def align_pairs_dropin(self, r1, r2, write_bam: int = 1) -> float:
        """The drop-in call hera's worker makes (hera_gpu_align_pairs:
        read_inf in, malloc'd Candidates out); the Candidates are freed
        afterwards as hera's destroy_candidate would.  Returns the call's
        wall milliseconds (the free excluded)."""
        a, ba = self._read_infs(r1)
        b, bb = self._read_infs(r2)
        out = np.zeros(2 * r1.n, np.uint64)
        self.lib.hera_gpu_align_pairs.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int,
                                                  C.c_void_p]
        self.lib.hera_gpu_free_candidates.argtypes = [C.c_void_p, C.c_int64]
        t0 = time.perf_counter()
        rc = self.lib.hera_gpu_align_pairs(self.h, _ptr(a), _ptr(b), r1.n, write_bam, _ptr(out))
        ms = (time.perf_counter() - t0) * 1e3
        self.lib.hera_gpu_free_candidates(_ptr(out), out.shape[0])
        self._check(rc)
        return ms

    def bgzf(self, data) -> tuple:
        """(BGZF bytes, device ms) of a byte buffer (hera_gpu_bgzf)."""
        a = np.frombuffer(data, np.uint8) if not isinstance(data, np.ndarray) else data
        a = np.ascontiguousarray(a, np.uint8)
        cap = a.size + (a.size // 0xff00 + 1) * 64 + 64
        out = np.empty(cap, np.uint8)
        used, ms = C.c_uint64(), C.c_float()
        self.lib.hera_gpu_bgzf.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
                                           C.POINTER(C.c_uint64), C.POINTER(C.c_float)]
        self._check(self.lib.hera_gpu_bgzf(self.h, _ptr(a) if a.size else None, a.size, _ptr(out), cap,
                                           C.byref(used), C.byref(ms)))
        return out[:used.value], ms.value

    def fetch(self, n_recs: int) -> Result:
        res = Result(n_recs, n_recs * 8 + 1024, n_recs * 8 + 1024, n_recs * 8 + 1024)
        rc = self.lib.hera_gpu_fetch_result(self.h, C.byref(res.c))
        if rc == -5:
            res._alloc(res.c.list_used + 1, res.c.op_used + 1, res.c.miss_used + 1)
            rc = self.lib.hera_gpu_fetch_result(self.h, C.byref(res.c))
        self._check(rc)
        return res

    def timing(self) -> dict:
        t = Timing()
        self.lib.hera_gpu_get_timing(self.h, C.byref(t))
        return t.as_dict()

    def tuning(self) -> dict:
        """Launch shapes in use and the autotuner's trial timings."""
        t = Tuning()
        self._check(self.lib.hera_gpu_get_tuning(self.h, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, build_blocks_per_sm: int, rescue_warps_per_block: int) -> None:
        """Pin the launch shapes (the autotuner then stays off)."""
        t = Tuning()
        t.build_blocks_per_sm, t.rescue_warps_per_block = build_blocks_per_sm, rescue_warps_per_block
        self._check(self.lib.hera_gpu_set_tuning(self.h, C.byref(t)))

    @property
    def stream(self) -> int:
        return self.lib.hera_gpu_stream(self.h) or 0

    # ---- FASTQ chunks -------------------------------------------------------

    @staticmethod
    def _chunk(b) -> np.ndarray:
        a = np.frombuffer(b, np.uint8) if isinstance(b, (bytes, bytearray, memoryview)) else b
        return np.ascontiguousarray(a, np.uint8)

    def _fastq_check(self, rc: int, bf: int, br: int) -> None:
        if rc == HERA_GPU_EFORMAT:
            raise FastqFormatError(rc, self.lib.hera_gpu_last_error(self.h).decode(), bf, br)
        self._check(rc)

    def parse_fastq_pairs(self, left, right) -> np.ndarray:
        """Reads of a pair of FASTQ chunk buffers (bytes or uint8 arrays),
        parsed on the device: FQ_DTYPE records, mates interleaved."""
        lb, rb = self._chunk(left), self._chunk(right)
        cap = max(16, min(lb.size, rb.size) // 64 + 16)
        while True:
            recs = np.empty(2 * cap, FQ_DTYPE)
            n, bf, br = C.c_int32(), C.c_int32(), C.c_int64()
            rc = self.lib.hera_gpu_parse_fastq_pairs(self.h, _ptr(lb) if lb.size else None, lb.size,
                                                     _ptr(rb) if rb.size else None, rb.size, _ptr(recs), cap,
                                                     C.byref(n), C.byref(bf), C.byref(br))
            if rc == HERA_GPU_ECAPACITY and n.value > cap:
                cap = n.value
                continue
            self._fastq_check(rc, bf.value, br.value)
            return recs[:2 * n.value]

    def parse_fastq_single(self, chunk) -> np.ndarray:
        b = self._chunk(chunk)
        cap = max(16, b.size // 64 + 16)
        while True:
            recs = np.empty(cap, FQ_DTYPE)
            n, br = C.c_int32(), C.c_int64()
            rc = self.lib.hera_gpu_parse_fastq_single(self.h, _ptr(b) if b.size else None, b.size, _ptr(recs),
                                                      cap, C.byref(n), C.byref(br))
            if rc == HERA_GPU_ECAPACITY and n.value > cap:
                cap = n.value
                continue
            self._fastq_check(rc, 1, br.value)
            return recs[:n.value]

    def align_fastq_pairs(self, left, right, write_bam: int = 1, out: Optional[Result] = None):
        """Parse a pair of FASTQ chunk buffers and align their pairs, all on
        the device: (Result, FQ_DTYPE records).  `out`: a Result to reuse
        (its storage is overwritten); the records array is reused between
        calls too (copy it to keep it)."""
        lb, rb = self._chunk(left), self._chunk(right)
        cap = max(16, min(lb.size, rb.size) // 64 + 16)
        while True:
            if getattr(self, "_fq_recs", None) is None or self._fq_recs.shape[0] < 2 * cap:
                self._fq_recs = np.empty(2 * cap, FQ_DTYPE)
            recs = self._fq_recs
            if out is not None:
                res = out.reuse(2 * cap)
            else:
                res = Result(2 * cap, 8 * cap + 1024, 8 * cap + 1024, (lb.size + rb.size) // 8 + 1024)
            n, bf, br = C.c_int32(), C.c_int32(), C.c_int64()
            rc = self.lib.hera_gpu_align_fastq_pairs(self.h, _ptr(lb) if lb.size else None, lb.size,
                                                     _ptr(rb) if rb.size else None, rb.size, write_bam,
                                                     _ptr(recs), cap, C.byref(n), C.byref(bf), C.byref(br),
                                                     C.byref(res.c))
            if rc == HERA_GPU_ECAPACITY and n.value > cap:
                cap = n.value
                continue
            if rc == HERA_GPU_ECAPACITY:   # result pools: fetch again into bigger ones
                res._alloc(res.c.list_used + 1, res.c.op_used + 1, res.c.miss_used + 1)
                rc = self.lib.hera_gpu_fetch_result(self.h, C.byref(res.c))
            self._fastq_check(rc, bf.value, br.value)
            res.recs = res._rec_buf[:2 * n.value]
            return res, recs[:2 * n.value]

    def fastq_stats(self) -> dict:
        s = FastqStats()
        self._check(self.lib.hera_gpu_get_fastq_stats(self.h, C.byref(s)))
        return s.as_dict()


class FastqReads:
    """A read set (seq, off, len) over a FASTQ chunk buffer for the records
    `recs` of it -- e.g. recs[0::2] of a pair's file 1 -- to pass to
    Context.align_pairs / align_single without copying the sequences."""

    def __init__(self, chunk, recs: np.ndarray):
        self.seq = Context._chunk(chunk)
        self.off = np.ascontiguousarray(recs["seq"], np.int64)
        self.len = np.ascontiguousarray(recs["len"], np.int32)

    @property
    def n(self) -> int:
        return int(self.len.shape[0])


class Server:
    """The serving loop of the C ABI (hera_gpu_server_*): chunks of read
    pairs from many samples, continuously batched onto device slots sized by
    free HBM, per-sample counters on the device."""

    def __init__(self, ctx: "Context", batch_pairs: int = 0, max_slots: int = 0, write_bam: int = 1,
                 max_samples: int = 0, hbm_reserve: int = 0, borrow_reads: bool = False):
        """borrow_reads: submit keeps pointers to the caller's reads (no
        copy); they must stay alive and unchanged until the chunk's wait."""
        self.ctx = ctx
        self.lib = ctx.lib
        opt = _ServerOptions(batch_pairs, max_slots, hbm_reserve, write_bam, max_samples, 1 if borrow_reads else 0)
        h = C.c_void_p()
        ctx._check(self.lib.hera_gpu_server_create(ctx.h, C.byref(opt), C.byref(h)))
        self.h = h
        self._sizes = {}

    def submit(self, sample: int, r1, r2) -> int:
        """Queue the pairs (r1[i], r2[i]) of `sample`; returns a ticket."""
        a, b = Context._reads(r1), Context._reads(r2)
        t = C.c_uint64()
        self.ctx._check(self.lib.hera_gpu_server_submit(self.h, sample, C.byref(a), C.byref(b), r1.n,
                                                        C.byref(t)))
        self._sizes[t.value] = (r1.n, int(r1.len.sum()) + int(r2.len.sum()))
        return t.value

    def wait(self, ticket: int, out: Optional[Result] = None):
        """(Result, info) of a chunk, blocking until it is done.  `out`: a
        Result to reuse (its storage is overwritten)."""
        n, total_len = self._sizes.pop(ticket)
        res = out.reuse(2 * n) if out is not None else Result(2 * n, 8 * n + 1024, 8 * n + 1024,
                                                               total_len // 8 + 1024)
        info = ChunkInfo()
        rc = self.lib.hera_gpu_server_wait(self.h, ticket, C.byref(res.c), C.byref(info))
        if rc == -5 and (res.c.list_used > res.c.list_cap or res.c.op_used > res.c.op_cap
                         or res.c.miss_used > res.c.miss_cap):
            res._alloc(res.c.list_used + 1, res.c.op_used + 1, res.c.miss_used + 1)
            rc = self.lib.hera_gpu_server_wait(self.h, ticket, C.byref(res.c), C.byref(info))
        self.ctx._check(rc)
        return res, info.as_dict()

    def cancel(self, sample: int) -> int:
        """Drop the sample's queued work; returns the chunks cancelled."""
        k = C.c_int32(0)
        self.lib.hera_gpu_server_cancel.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(C.c_int32)]
        self.ctx._check(self.lib.hera_gpu_server_cancel(self.h, sample, C.byref(k)))
        return k.value

    def sample_stats(self, sample: int) -> dict:
        st = SampleStats()
        self.ctx._check(self.lib.hera_gpu_server_get_sample_stats(self.h, sample, C.byref(st)))
        return st.as_dict()

    def stats(self) -> dict:
        st = ServerStats()
        self.ctx._check(self.lib.hera_gpu_server_get_stats(self.h, C.byref(st)))
        return st.as_dict()

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.hera_gpu_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tally(res: Result) -> dict:
    """The per-sample counters the server keeps on the device, computed on
    the host from one chunk's records (for checking)."""
    r = res.recs
    a, b = r[0::2], r[1::2]
    hits = a["n"].sum(axis=1).astype(np.int64) + b["n"].sum(axis=1)
    return {"pairs": int(a.shape[0]), "mapped": int((hits > 0).sum()), "paired": int((a["pair"] == 2).sum()),
            "hits": int(hits.sum()),
            "cigar_ops": int(a["n_cigar"].astype(np.int64).sum() + b["n_cigar"].astype(np.int64).sum())}


class ClassTable:
    """A class table copied off the device: hera's CLASS (classes in
    first-insertion order: XXH32 id, read count, transcript list),
    REF_INF->count, PAIRED and MEAN_FRAG's running sum."""

    def __init__(self, ids, counts, ns, list_off, lists, tx_count, paired, mean_frag):
        self.ids, self.counts, self.ns = ids, counts, ns
        self.ref_off, self.ref, self.tx_count = list_off, lists, tx_count
        self.paired, self.mean_frag = int(paired), float(mean_frag)

    @property
    def n_classes(self) -> int:
        return len(self.ids)

    def lists(self):
        return [tuple(self.ref[int(o):int(o) + int(n)]) for o, n in zip(self.ref_off, self.ns)]

    def key(self):
        """Everything hera's EM and summary read, as plain values."""
        return (tuple(self.ids.tolist()), tuple(self.counts.tolist()), tuple(self.lists()),
                tuple(self.tx_count.tolist()), self.paired, self.mean_frag)


class Classes:
    """hera's add_class (src/hash_align.c:1564-1602) on the device: one class
    table that the records of a run are added to batch by batch, in input
    order.  A context's device-resident results go in with add_last(),
    records already in device memory with add_device()."""

    def __init__(self, ctx: "Context", max_classes: int = 1 << 20, max_list: int = 1 << 24):
        self.lib = ctx.lib
        self.n_trans = ctx.index.n_trans
        h = C.c_void_p()
        ctx._check(self.lib.hera_gpu_classes_create(ctx.h, max_classes, max_list, C.byref(h)))
        self.h = h

    def _check(self, rc: int) -> None:
        if rc != HERA_GPU_OK:
            raise HeraGpuError(rc, self.lib.hera_gpu_classes_last_error(self.h).decode())

    def add_last(self, ctx: "Context") -> None:
        """The pairs of ctx's last align_pairs_device call."""
        self._check(self.lib.hera_gpu_classes_add_last(self.h, ctx.h))

    def add_device(self, d_recs: int, d_pos_pool: int, d_p_pool: int, n: int, paired: bool = True,
                   stream: Optional[int] = None) -> None:
        self._check(self.lib.hera_gpu_classes_add_device(self.h, d_recs, d_pos_pool, d_p_pool, n,
                                                         1 if paired else 0, stream))

    def add_result(self, res: "Result", paired: bool = True) -> None:
        """Records in host memory (a Result from an align call or a server
        wait), copied to the device and added."""
        n = res.recs.shape[0] // 2 if paired else res.recs.shape[0]
        self._check(self.lib.hera_gpu_classes_add_host(self.h, C.byref(res.c), n, 1 if paired else 0))

    def load(self, table) -> None:
        """Replace the contents with a class table held on the host (any
        object with ids, counts, ns, ref_off, ref, tx_count, paired and
        mean_frag, e.g. a ClassTable)."""
        keep = [np.ascontiguousarray(table.ids, np.uint32), np.ascontiguousarray(table.counts, np.float64),
                np.ascontiguousarray(table.ns, np.uint32), np.ascontiguousarray(table.ref_off, np.uint64),
                np.ascontiguousarray(np.append(np.asarray(table.ref, np.uint32), np.uint32(0))),
                np.ascontiguousarray(table.tx_count, np.uint32)]
        ids, cnt, ns, offs, ref, tx = keep
        t = _ClassTable()
        t.class_cap = t.n_classes = len(ids)
        t.id, t.count, t.n, t.list_off = _ptr(ids), _ptr(cnt), _ptr(ns), _ptr(offs)
        t.list_cap = t.list_used = len(ref) - 1
        t.list, t.tx_count = _ptr(ref), _ptr(tx)
        t.paired, t.mean_frag_sum = int(table.paired), float(table.mean_frag)
        self._check(self.lib.hera_gpu_classes_load(self.h, C.byref(t)))

    def em(self, ctx: "Context"):
        """hera's estimate_count on the device over this table:
        (grama, overlap, rounds, device ms), the arrays bit for bit as hera's
        em_val leaves them."""
        n = self.n_trans
        g, o = np.zeros(max(n, 1)), np.zeros(max(n, 1))
        rounds, ms = C.c_uint32(), C.c_float()
        self._check(self.lib.hera_gpu_classes_em(self.h, ctx.h, _ptr(g), _ptr(o), C.byref(rounds), C.byref(ms)))
        return g[:n], o[:n], rounds.value, ms.value

    def timing(self) -> dict:
        ms, n = C.c_float(), C.c_uint32()
        self.lib.hera_gpu_classes_timing(self.h, C.byref(ms), C.byref(n))
        return {"kernel_ms": ms.value, "launches": n.value}

    def fetch(self) -> ClassTable:
        t = _ClassTable()
        rc = self.lib.hera_gpu_classes_fetch(self.h, C.byref(t))
        if rc != HERA_GPU_OK and rc != HERA_GPU_ECAPACITY:
            self._check(rc)
        nc, nl = t.n_classes, t.list_used
        ids = np.zeros(max(nc, 1), np.uint32)
        counts = np.zeros(max(nc, 1), np.float64)
        ns = np.zeros(max(nc, 1), np.uint32)
        offs = np.zeros(max(nc, 1), np.uint64)
        lists = np.zeros(max(nl, 1), np.uint32)
        tx = np.zeros(max(self.n_trans, 1), np.uint32)
        t.class_cap, t.list_cap = nc, nl
        t.id, t.count, t.n, t.list_off = _ptr(ids), _ptr(counts), _ptr(ns), _ptr(offs)
        t.list, t.tx_count = _ptr(lists), _ptr(tx)
        self._check(self.lib.hera_gpu_classes_fetch(self.h, C.byref(t)))
        return ClassTable(ids[:nc], counts[:nc], ns[:nc], offs[:nc], lists[:nl], tx[:self.n_trans],
                          t.paired, t.mean_frag_sum)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.hera_gpu_classes_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BamWriter:
    """The tail's BAM records (`-w`) on the device: hera_gpu_bam_pairs.
    `gene_map`: any object with chr_len, exon_off, starts, ends, chr and
    gene arrays (hera's GENE_MAP)."""

    def __init__(self, ctx: "Context", gene_map):
        self.lib = ctx.lib
        self._gm = [np.ascontiguousarray(getattr(gene_map, k), np.uint32)
                    for k in ("chr_len", "exon_off", "starts", "ends", "chr", "gene")]
        g = _GeneMap(len(self._gm[0]), *[_ptr(a) for a in self._gm])
        h = C.c_void_p()
        ctx._check(self.lib.hera_gpu_bam_create(ctx.h, C.byref(g), C.byref(h)))
        self.h = h

    def pairs(self, res: "Result", r1, r2, qual1: np.ndarray, qual2: np.ndarray, names1: np.ndarray,
              names2: np.ndarray, cap: int = 0):
        """(bytes, per-pair offsets, device ms) of the records of r1.n pairs;
        names: (n, stride) uint8 arrays, NUL-terminated rows."""
        n = r1.n
        a, b = Context._reads(r1), Context._reads(r2)
        cap = cap or int(r1.len.sum() + r2.len.sum()) * 8 + 4096 * n + 4096
        out = np.zeros(cap, np.uint8)
        off = np.zeros(n + 1, np.uint64)
        ms = C.c_float()
        args = (self.h, C.byref(res.c), n, C.byref(a), C.byref(b), _ptr(qual1), _ptr(qual2), _ptr(names1),
                _ptr(names2), names1.shape[1])
        rc = self.lib.hera_gpu_bam_pairs(*args, _ptr(out), cap, _ptr(off), C.byref(ms))
        if rc == HERA_GPU_ECAPACITY and int(off[-1]) > cap:
            cap = int(off[-1])
            out = np.zeros(cap, np.uint8)
            rc = self.lib.hera_gpu_bam_pairs(*args, _ptr(out), cap, _ptr(off), C.byref(ms))
        if rc != HERA_GPU_OK:
            raise HeraGpuError(rc, self.lib.hera_gpu_bam_last_error(self.h).decode())
        return out[:int(off[-1])], off, ms.value

    def single(self, res: "Result", rs, qual: np.ndarray, names: np.ndarray, cap: int = 0):
        """(bytes, per-read offsets, device ms) of the records of rs.n single
        reads (align_single_read's writes)."""
        n = rs.n
        a = Context._reads(rs)
        cap = cap or int(rs.len.sum()) * 8 + 4096 * n + 4096
        out = np.zeros(cap, np.uint8)
        off = np.zeros(n + 1, np.uint64)
        ms = C.c_float()
        self.lib.hera_gpu_bam_single.argtypes = [C.c_void_p, C.POINTER(_Result), C.c_int32, C.POINTER(_Reads),
                                                 C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_uint64,
                                                 C.c_void_p, C.POINTER(C.c_float)]
        args = (self.h, C.byref(res.c), n, C.byref(a), _ptr(qual), _ptr(names), names.shape[1])
        rc = self.lib.hera_gpu_bam_single(*args, _ptr(out), cap, _ptr(off), C.byref(ms))
        if rc == HERA_GPU_ECAPACITY and int(off[-1]) > cap:
            cap = int(off[-1])
            out = np.zeros(cap, np.uint8)
            rc = self.lib.hera_gpu_bam_single(*args, _ptr(out), cap, _ptr(off), C.byref(ms))
        if rc != HERA_GPU_OK:
            raise HeraGpuError(rc, self.lib.hera_gpu_bam_last_error(self.h).decode())
        return out[:int(off[-1])], off, ms.value

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.hera_gpu_bam_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
