"""sadcs_b200: suffix array and BWT construction on one B200, in hand-written sm_100a CUDA kernels.

The Python side mirrors the reference's GPU interface (src/cuda/gpusa.h of acesds/sadcs) over the
C ABI of ``lib/libsadcs_gpu.so`` (include/sadcs_gpu.h):

=========================  =====================================  ===========================
here                       C ABI                                  reference (gpusa.h)
=========================  =====================================  ===========================
``query_device()``         ``sadcs_gpu_query_device``             ``gpuQueryDevice`` :76
``required_bytes(n)``      ``sadcs_gpu_required_bytes``           ``gpuRequiredBytes`` :79
``sample_size(n)``         ``sadcs_gpu_sample_size``              ``gpuSampleSize`` :57-60
``Context(capacity)``      ``sadcs_gpu_create/destroy_context``   ``gpuCreateContext`` :93, :96
``suffix_array(text)``     ``sadcs_gpu_suffix_array``             ``gpuSuffixArray`` :102-103
``bwt(text)``              ``sadcs_gpu_bwt``                      ``gpuBwt`` :108-109
``rank_sample(text)``      ``sadcs_gpu_rank_sample``              ``gpuRankSample`` :115
``allocate_pinned(n)``     ``sadcs_gpu_allocate_pinned``          ``gpuAllocatePinned`` :120
``build(text)``            ``sadcs_gpu_build``                    (no counterpart: SA + BWT)
``build_device(...)``      ``sadcs_gpu_build_device``             (no counterpart)
``bwt_from_sa_device``     ``sadcs_gpu_bwt_from_sa``              (no counterpart)
=========================  =====================================  ===========================

Statuses are GpuStatus's (Ok, Unavailable, NotEnoughMemory, Failed); a status other than Ok raises
``GpuError`` carrying it and ``sadcs_gpu_last_error()``. There is no CPU fallback: without the
library, importing the bindings raises.
"""
from __future__ import annotations

import ctypes
import enum
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "lib" / "libsadcs_gpu.so"


class GpuStatus(enum.IntEnum):
    Ok = 0
    Unavailable = 1
    NotEnoughMemory = 2
    Failed = 3


class GpuError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = GpuStatus(status)
        super().__init__(f"{self.status.name}: {message}")


class Device(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 256), ("compute_major", ctypes.c_int32), ("compute_minor", ctypes.c_int32),
                ("total_bytes", ctypes.c_int64), ("free_bytes", ctypes.c_int64)]


class Stats(ctypes.Structure):
    """GpuStats (gpusa.h:37-53)."""
    _fields_ = [("device_bytes", ctypes.c_int64), ("ranking_bytes", ctypes.c_int64),
                ("class_sort_bytes", ctypes.c_int64), ("merge_bytes", ctypes.c_int64),
                ("pinned", ctypes.c_int32), ("character_passes", ctypes.c_int32),
                ("doubling_rounds", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("setup_seconds", ctypes.c_double), ("upload_seconds", ctypes.c_double),
                ("device_seconds", ctypes.c_double), ("ranking_seconds", ctypes.c_double),
                ("class_sort_seconds", ctypes.c_double), ("merge_seconds", ctypes.c_double),
                ("bwt_seconds", ctypes.c_double), ("download_seconds", ctypes.c_double),
                ("ranking_device_ms", ctypes.c_double), ("class_sort_device_ms", ctypes.c_double),
                ("merge_device_ms", ctypes.c_double), ("merge_kernel_ms", ctypes.c_double),
                ("kernel_launches", ctypes.c_int64)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_ctxp = ctypes.c_void_p

_lib = None


def library_path() -> Path:
    return _LIB_PATH


def lib() -> ctypes.CDLL:
    """The C ABI. Raises if libsadcs_gpu.so was not built: there is no fallback."""
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise ImportError(f"{_LIB_PATH} is missing: build it with `python -m sadcs_b200.build` "
                              "(nvcc, sm_100a); there is no CPU fallback")
        L = ctypes.CDLL(str(_LIB_PATH))
        L.sadcs_gpu_memory_reserve.restype = ctypes.c_int64
        L.sadcs_gpu_memory_reserve.argtypes = []
        L.sadcs_gpu_sample_size.restype = ctypes.c_int64
        L.sadcs_gpu_sample_size.argtypes = [ctypes.c_int64]
        L.sadcs_gpu_query_device.restype = ctypes.c_int
        L.sadcs_gpu_query_device.argtypes = [ctypes.POINTER(Device)]
        L.sadcs_gpu_required_bytes.restype = ctypes.c_int64
        L.sadcs_gpu_required_bytes.argtypes = [ctypes.c_int64]
        L.sadcs_gpu_create_context.restype = ctypes.c_int
        L.sadcs_gpu_create_context.argtypes = [ctypes.c_int64, ctypes.POINTER(_ctxp)]
        L.sadcs_gpu_destroy_context.restype = None
        L.sadcs_gpu_destroy_context.argtypes = [_ctxp]
        L.sadcs_gpu_context_capacity.restype = ctypes.c_int64
        L.sadcs_gpu_context_capacity.argtypes = [_ctxp]
        L.sadcs_gpu_suffix_array.restype = ctypes.c_int
        L.sadcs_gpu_suffix_array.argtypes = [_ctxp, _u8p, ctypes.c_int64, _i32p, ctypes.POINTER(Stats)]
        L.sadcs_gpu_bwt.restype = ctypes.c_int
        L.sadcs_gpu_bwt.argtypes = [_ctxp, _u8p, ctypes.c_int64, _u8p, _i32p, ctypes.POINTER(Stats)]
        L.sadcs_gpu_rank_sample.restype = ctypes.c_int
        L.sadcs_gpu_rank_sample.argtypes = [_u8p, ctypes.c_int64, _u32p, ctypes.POINTER(Stats)]
        L.sadcs_gpu_allocate_pinned.restype = ctypes.c_void_p
        L.sadcs_gpu_allocate_pinned.argtypes = [ctypes.c_size_t]
        L.sadcs_gpu_free_pinned.restype = None
        L.sadcs_gpu_free_pinned.argtypes = [ctypes.c_void_p]
        L.sadcs_gpu_last_error.restype = ctypes.c_char_p
        L.sadcs_gpu_last_error.argtypes = []
        L.sadcs_gpu_build.restype = ctypes.c_int
        L.sadcs_gpu_build.argtypes = [_ctxp, _u8p, ctypes.c_int64, _u32p, _u8p, _i64p, ctypes.POINTER(Stats)]
        L.sadcs_gpu_build_device.restype = ctypes.c_int
        L.sadcs_gpu_build_device.argtypes = [_ctxp, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                             ctypes.c_void_p, _i64p, ctypes.c_void_p, ctypes.POINTER(Stats)]
        L.sadcs_gpu_bwt_from_sa.restype = ctypes.c_int
        L.sadcs_gpu_bwt_from_sa.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                            _i64p, ctypes.c_void_p]
        L.sadcs_gpu_required_bytes_batch.restype = ctypes.c_int64
        L.sadcs_gpu_required_bytes_batch.argtypes = [ctypes.c_int64, ctypes.c_int64]
        L.sadcs_gpu_create_batch_context.restype = ctypes.c_int
        L.sadcs_gpu_create_batch_context.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.POINTER(_ctxp)]
        L.sadcs_gpu_build_batch.restype = ctypes.c_int
        L.sadcs_gpu_build_batch.argtypes = [_ctxp, _u8p, _i64p, ctypes.c_int64, _u32p, _u8p, _i64p,
                                            ctypes.POINTER(Stats)]
        L.sadcs_gpu_build_batch_device.restype = ctypes.c_int
        L.sadcs_gpu_build_batch_device.argtypes = [_ctxp, ctypes.c_void_p, _i64p, ctypes.c_int64, ctypes.c_void_p,
                                                   ctypes.c_void_p, _i64p, ctypes.c_void_p, ctypes.POINTER(Stats)]
        L.sadcs_gpu_server_create.restype = ctypes.c_int
        L.sadcs_gpu_server_create.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64,
                                              ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]
        L.sadcs_gpu_server_submit.restype = ctypes.c_int
        L.sadcs_gpu_server_submit.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_int64, _u32p, _u8p,
                                              ctypes.POINTER(ctypes.c_uint64)]
        L.sadcs_gpu_server_wait.restype = ctypes.c_int
        L.sadcs_gpu_server_wait.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double, _i64p,
                                            ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32)]
        L.sadcs_gpu_server_counters.restype = None
        L.sadcs_gpu_server_counters.argtypes = [ctypes.c_void_p, _i64p, _i64p]
        L.sadcs_gpu_server_destroy.restype = None
        L.sadcs_gpu_server_destroy.argtypes = [ctypes.c_void_p]
        L.sadcs_gpu_server_cancel.restype = ctypes.c_int
        L.sadcs_gpu_server_cancel.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
        L.sadcs_gpu_server_fail_allocations.restype = None
        L.sadcs_gpu_server_fail_allocations.argtypes = [ctypes.c_void_p, ctypes.c_int64]
        L.sadcs_gpu_check_bwt.restype = ctypes.c_int
        L.sadcs_gpu_check_bwt.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, _i64p,
                                          ctypes.c_void_p]
        L.sadcs_gpu_inverse_bwt.restype = ctypes.c_int
        L.sadcs_gpu_inverse_bwt.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
                                            ctypes.c_void_p]
        L.sadcs_gpu_check_suffix_array.restype = ctypes.c_int
        L.sadcs_gpu_check_suffix_array.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, _i64p,
                                                   ctypes.POINTER(ctypes.c_char_p), ctypes.c_void_p]
        L.sadcs_gpu_check_suffix_array_static.restype = ctypes.c_int
        L.sadcs_gpu_check_suffix_array_static.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, _i64p,
                                                          ctypes.POINTER(ctypes.c_char_p), ctypes.c_void_p]
        L.sadcs_gpu_check_suffix_array_host.restype = ctypes.c_int
        L.sadcs_gpu_check_suffix_array_host.argtypes = [_u8p, ctypes.c_int64, _u32p, _i64p,
                                                        ctypes.POINTER(ctypes.c_char_p)]
        L.sadcs_gpu_check_bwt_host.restype = ctypes.c_int
        L.sadcs_gpu_check_bwt_host.argtypes = [_u8p, ctypes.c_int64, _u8p, ctypes.c_int64, _i64p]
        L.sadcs_gpu_test_lookback_timeout.restype = ctypes.c_int
        L.sadcs_gpu_test_lookback_timeout.argtypes = [ctypes.c_int64, _u32p]
        L.sadcs_gpu_lcp.restype = ctypes.c_int
        L.sadcs_gpu_lcp.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        _lib = L
    return _lib


def last_error() -> str:
    return lib().sadcs_gpu_last_error().decode(errors="replace")


def _check(status: int) -> None:
    if status != GpuStatus.Ok:
        raise GpuError(status, last_error())


def _as_text(text) -> np.ndarray:
    if isinstance(text, (bytes, bytearray, memoryview)):
        a = np.frombuffer(bytes(text), dtype=np.uint8)
    else:
        a = np.asarray(text)
        if a.dtype != np.uint8:
            raise TypeError(f"text must be uint8 bytes, got {a.dtype}")
    return np.ascontiguousarray(a)


def sample_size(n: int) -> int:
    return int(lib().sadcs_gpu_sample_size(n))


def memory_reserve() -> int:
    return int(lib().sadcs_gpu_memory_reserve())


def required_bytes(n: int) -> int:
    return int(lib().sadcs_gpu_required_bytes(n))


def query_device() -> dict:
    d = Device()
    _check(lib().sadcs_gpu_query_device(ctypes.byref(d)))
    return {"name": d.name.decode(), "compute": (d.compute_major, d.compute_minor),
            "total_bytes": d.total_bytes, "free_bytes": d.free_bytes}


class Context:
    """Device memory for texts of up to ``capacity`` bytes, reserved once (gpuCreateContext).
    ``max_texts`` > 1 makes a batch context: batches of up to that many texts of ``capacity``
    bytes together."""

    def __init__(self, capacity: int, max_texts: int = 1):
        handle = _ctxp()
        if max_texts == 1:
            _check(lib().sadcs_gpu_create_context(int(capacity), ctypes.byref(handle)))
        else:
            _check(lib().sadcs_gpu_create_batch_context(int(capacity), int(max_texts), ctypes.byref(handle)))
        self._handle = handle

    @property
    def handle(self):
        return self._handle

    @property
    def capacity(self) -> int:
        return int(lib().sadcs_gpu_context_capacity(self._handle))

    def close(self) -> None:
        if getattr(self, "_handle", None):
            lib().sadcs_gpu_destroy_context(self._handle)
            self._handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _handle(context):
    return context.handle if context is not None else None


def suffix_array(text, context: Context | None = None, stats: Stats | None = None) -> np.ndarray:
    """gpuSuffixArray: the int32 suffix array of text (n <= 2^31 - 1025)."""
    t = _as_text(text)
    n = len(t)
    sa = np.empty(max(n, 1), np.int32)
    _check(lib().sadcs_gpu_suffix_array(_handle(context), t.ctypes.data_as(_u8p), n, sa.ctypes.data_as(_i32p),
                                        ctypes.byref(stats) if stats is not None else None))
    return sa[:n]


def bwt(text, context: Context | None = None, stats: Stats | None = None):
    """gpuBwt: (BWT bytes, primary index) of text."""
    t = _as_text(text)
    n = len(t)
    out = np.empty(max(n, 1), np.uint8)
    primary = ctypes.c_int32(-1)
    _check(lib().sadcs_gpu_bwt(_handle(context), t.ctypes.data_as(_u8p), n, out.ctypes.data_as(_u8p),
                               ctypes.byref(primary), ctypes.byref(stats) if stats is not None else None))
    return out[:n], int(primary.value)


def rank_sample(text, stats: Stats | None = None) -> np.ndarray:
    """gpuRankSample: ranks of the sample suffixes (cover mod 32), gpuSampleSize(n) entries."""
    t = _as_text(text)
    n = len(t)
    ranks = np.empty(max(sample_size(n), 1), np.uint32)
    _check(lib().sadcs_gpu_rank_sample(t.ctypes.data_as(_u8p), n, ranks.ctypes.data_as(_u32p),
                                       ctypes.byref(stats) if stats is not None else None))
    return ranks[:sample_size(n)]


def build(text, want_sa: bool = True, want_bwt: bool = True, context: Context | None = None,
          stats: Stats | None = None, out_sa: np.ndarray | None = None, out_bwt: np.ndarray | None = None):
    """SA (uint32) and/or BWT from one construction, host to host, n up to 2^32 - 256. out_sa /
    out_bwt may be given as the output buffers (page-locked ones are written by the device directly).

    Returns (sa or None, bwt or None, primary or None)."""
    t = _as_text(text)
    n = len(t)
    sa = (out_sa if out_sa is not None else np.empty(max(n, 1), np.uint32)) if want_sa else None
    out = (out_bwt if out_bwt is not None else np.empty(max(n, 1), np.uint8)) if want_bwt else None
    if (sa is not None and (sa.dtype != np.uint32 or len(sa) < n)) or (out is not None and (out.dtype != np.uint8 or len(out) < n)):
        raise ValueError("out_sa must be uint32 and out_bwt uint8, each of at least n entries")
    primary = ctypes.c_int64(-1)
    _check(lib().sadcs_gpu_build(_handle(context), t.ctypes.data_as(_u8p), n,
                                 sa.ctypes.data_as(_u32p) if sa is not None else None,
                                 out.ctypes.data_as(_u8p) if out is not None else None, ctypes.byref(primary),
                                 ctypes.byref(stats) if stats is not None else None))
    return (sa[:n] if sa is not None else None, out[:n] if out is not None else None,
            int(primary.value) if want_bwt else None)


def required_bytes_batch(total: int, texts: int) -> int:
    return int(lib().sadcs_gpu_required_bytes_batch(int(total), int(texts)))


def build_batch(texts, want_sa: bool = True, want_bwt: bool = True, context: Context | None = None,
                stats: Stats | None = None, out_sa: np.ndarray | None = None, out_bwt: np.ndarray | None = None):
    """SA and/or BWT of every text of a list in one construction (sadcs_gpu_build_batch). out_sa /
    out_bwt may be given as the output buffers of all texts one after another (page-locked ones are
    filled while the construction runs).

    Returns (list of SA arrays or None, list of BWT arrays or None, list of primaries or None)."""
    arrays = [_as_text(t) for t in texts]
    lengths = np.array([len(a) for a in arrays], dtype=np.int64)
    packed = np.ascontiguousarray(np.concatenate(arrays) if arrays else np.zeros(0, np.uint8))
    total = int(lengths.sum())
    sa = (out_sa if out_sa is not None else np.empty(max(total, 1), np.uint32)) if want_sa else None
    out = (out_bwt if out_bwt is not None else np.empty(max(total, 1), np.uint8)) if want_bwt else None
    if (sa is not None and (sa.dtype != np.uint32 or len(sa) < total)) or (
            out is not None and (out.dtype != np.uint8 or len(out) < total)):
        raise ValueError("out_sa must be uint32 and out_bwt uint8, each of at least the texts' total length")
    primaries = np.zeros(max(len(arrays), 1), np.int64)
    _check(lib().sadcs_gpu_build_batch(_handle(context), packed.ctypes.data_as(_u8p) if packed.size else None,
                                       lengths.ctypes.data_as(_i64p), len(arrays),
                                       sa.ctypes.data_as(_u32p) if sa is not None else None,
                                       out.ctypes.data_as(_u8p) if out is not None else None,
                                       primaries.ctypes.data_as(_i64p),
                                       ctypes.byref(stats) if stats is not None else None))
    offsets = np.concatenate([[0], np.cumsum(lengths)])
    sas = [sa[offsets[j]:offsets[j + 1]] for j in range(len(arrays))] if want_sa else None
    bwts = [out[offsets[j]:offsets[j + 1]] for j in range(len(arrays))] if want_bwt else None
    return sas, bwts, ([int(p) for p in primaries[:len(arrays)]] if want_bwt else None)


def build_batch_device(d_texts: int, lengths, d_sa: int | None, d_bwt: int | None, context: Context | None = None,
                       stream: int | None = None, stats: Stats | None = None):
    """Device-resident batch: packed device texts, device outputs; returns the primaries."""
    lengths = np.ascontiguousarray(np.asarray(lengths, dtype=np.int64))
    primaries = np.zeros(max(len(lengths), 1), np.int64)
    _check(lib().sadcs_gpu_build_batch_device(_handle(context), ctypes.c_void_p(d_texts),
                                              lengths.ctypes.data_as(_i64p), len(lengths),
                                              ctypes.c_void_p(d_sa) if d_sa else None,
                                              ctypes.c_void_p(d_bwt) if d_bwt else None,
                                              primaries.ctypes.data_as(_i64p),
                                              ctypes.c_void_p(stream) if stream else None,
                                              ctypes.byref(stats) if stats is not None else None))
    return [int(p) for p in primaries[:len(lengths)]]


def build_device(d_text: int, n: int, d_sa: int | None, d_bwt: int | None, context: Context | None = None,
                 stream: int | None = None, stats: Stats | None = None) -> int:
    """Device-resident construction: raw device pointers (e.g. torch tensor data_ptr()), the caller's
    stream handle (cudaStream_t as int, 0/None for the legacy default stream). Returns the primary
    index (-1 when no BWT was asked for)."""
    primary = ctypes.c_int64(-1)
    _check(lib().sadcs_gpu_build_device(_handle(context), ctypes.c_void_p(d_text), int(n),
                                        ctypes.c_void_p(d_sa) if d_sa else None,
                                        ctypes.c_void_p(d_bwt) if d_bwt else None, ctypes.byref(primary),
                                        ctypes.c_void_p(stream) if stream else None,
                                        ctypes.byref(stats) if stats is not None else None))
    return int(primary.value)


def bwt_from_sa_device(d_text: int, n: int, d_sa: int, d_bwt: int, stream: int | None = None) -> int:
    """The SA-to-BWT gather on device buffers; returns the primary index."""
    primary = ctypes.c_int64(-1)
    _check(lib().sadcs_gpu_bwt_from_sa(ctypes.c_void_p(d_text), int(n), ctypes.c_void_p(d_sa),
                                       ctypes.c_void_p(d_bwt), ctypes.byref(primary),
                                       ctypes.c_void_p(stream) if stream else None))
    return int(primary.value)


def check_suffix_array_device(d_text: int, n: int, d_sa: int, stream: int | None = None):
    """The reference checker's fast mode on device buffers: (ok, first failing index, reason)."""
    index = ctypes.c_int64(-1)
    reason = ctypes.c_char_p()
    _check(lib().sadcs_gpu_check_suffix_array(ctypes.c_void_p(d_text), int(n), ctypes.c_void_p(d_sa),
                                              ctypes.byref(index), ctypes.byref(reason),
                                              ctypes.c_void_p(stream) if stream else None))
    return index.value < 0, int(index.value), reason.value.decode() if reason.value else None


STATIC_CHECK_MAX = 1 << 20  # SADCS_GPU_STATIC_CHECK_MAX


def check_suffix_array_static_device(d_text: int, n: int, d_sa: int, stream: int | None = None):
    """check_suffix_array_device without any allocation (sadcs_gpu_check_suffix_array_static): n up
    to STATIC_CHECK_MAX; calls on one device must not overlap in time."""
    index = ctypes.c_int64(-1)
    reason = ctypes.c_char_p()
    _check(lib().sadcs_gpu_check_suffix_array_static(ctypes.c_void_p(d_text), int(n), ctypes.c_void_p(d_sa),
                                                     ctypes.byref(index), ctypes.byref(reason),
                                                     ctypes.c_void_p(stream) if stream else None))
    return index.value < 0, int(index.value), reason.value.decode() if reason.value else None


def check_bwt_device(d_text: int, n: int, d_bwt: int, primary: int, stream: int | None = None):
    """The reference's BWT check on device buffers: (ok, first failing text position)."""
    index = ctypes.c_int64(-1)
    _check(lib().sadcs_gpu_check_bwt(ctypes.c_void_p(d_text), int(n), ctypes.c_void_p(d_bwt), int(primary),
                                     ctypes.byref(index), ctypes.c_void_p(stream) if stream else None))
    return index.value < 0, int(index.value)


def check_suffix_array(text, suffixes: np.ndarray):
    """checkSuffixArray in fast mode (src/common/checker.h:24) on host arrays, run on the device
    (sadcs_gpu_check_suffix_array_host): (ok, first failing SA index, reason)."""
    t = _as_text(text)
    s = np.ascontiguousarray(suffixes)
    if s.dtype not in (np.uint32, np.int32) or len(s) != len(t):
        raise ValueError("the suffix array must hold one 32-bit entry per text byte")
    index = ctypes.c_int64(-1)
    reason = ctypes.c_char_p()
    _check(lib().sadcs_gpu_check_suffix_array_host(t.ctypes.data_as(_u8p), len(t), s.ctypes.data_as(_u32p),
                                                   ctypes.byref(index), ctypes.byref(reason)))
    return index.value < 0, int(index.value), reason.value.decode() if reason.value else None


def check_bwt(text, bwt_bytes: np.ndarray, primary: int):
    """checkBwt (src/common/checker.h:29) on host arrays, run on the device
    (sadcs_gpu_check_bwt_host): (ok, first text position where the inverse differs)."""
    t = _as_text(text)
    b = _as_text(bwt_bytes)
    if len(b) != len(t):
        raise ValueError("the BWT must have as many bytes as the text")
    index = ctypes.c_int64(-1)
    _check(lib().sadcs_gpu_check_bwt_host(t.ctypes.data_as(_u8p), len(t), b.ctypes.data_as(_u8p), int(primary),
                                          ctypes.byref(index)))
    return index.value < 0, int(index.value)


def inverse_bwt_device(d_bwt: int, n: int, primary: int, d_text: int, stream: int | None = None) -> None:
    """unbwt on device buffers: d_text (n bytes) from the BWT and its primary index."""
    _check(lib().sadcs_gpu_inverse_bwt(ctypes.c_void_p(d_bwt), int(n), int(primary), ctypes.c_void_p(d_text),
                                       ctypes.c_void_p(stream) if stream else None))


def lcp_device(d_text: int, n: int, d_sa: int, d_lcp: int, stream: int | None = None) -> None:
    """The LCP array of a device suffix array (sadcs_gpu_lcp): d_lcp[0] = 0 and d_lcp[r] = the
    longest common prefix of suffixes d_sa[r - 1] and d_sa[r] (n uint32 entries; d_lcp may be d_sa)."""
    _check(lib().sadcs_gpu_lcp(ctypes.c_void_p(d_text), int(n), ctypes.c_void_p(d_sa), ctypes.c_void_p(d_lcp),
                               ctypes.c_void_p(stream) if stream else None))


def test_lookback_timeout(limit_cycles: int):
    """The radix look-back's time-out made to happen (sadcs_gpu_test_lookback_timeout): one pass
    whose only block waits on a status nothing publishes. Returns (status, error word, message)."""
    word = ctypes.c_uint32(0)
    status = lib().sadcs_gpu_test_lookback_timeout(int(limit_cycles), ctypes.byref(word))
    return GpuStatus(status), int(word.value), last_error()


def allocate_pinned(nbytes: int) -> np.ndarray:
    """Page-locked host memory as a uint8 array (freed with free_pinned)."""
    ptr = lib().sadcs_gpu_allocate_pinned(int(nbytes))
    if not ptr:
        raise MemoryError("cannot allocate page-locked host memory")
    buf = (ctypes.c_uint8 * max(int(nbytes), 1)).from_address(ptr)
    arr = np.frombuffer(buf, dtype=np.uint8, count=int(nbytes))
    return arr


def free_pinned(array: np.ndarray) -> None:
    lib().sadcs_gpu_free_pinned(ctypes.c_void_p(array.ctypes.data))


class Server:
    """The request loop of the library (sadcs_gpu_server_*): submit texts at any time, wait for
    their SA (uint32) and BWT. Queued small requests are built together in one batched
    construction; constructions of different workers overlap on the device; admission is by
    planned device footprint against ``memory_budget`` (<= 0: free memory minus the reserve)."""

    def __init__(self, memory_budget: int = 0, workers: int = 2, small_limit: int = 4 << 20,
                 batch_bytes: int = 256 << 20, batch_texts: int = 4096):
        handle = ctypes.c_void_p()
        _check(lib().sadcs_gpu_server_create(int(memory_budget), int(workers), int(small_limit), int(batch_bytes),
                                             int(batch_texts), ctypes.byref(handle)))
        self._handle = handle
        self._pending = {}

    def submit(self, text, sa: np.ndarray | None = None, bwt: np.ndarray | None = None) -> int:
        """Queues a text; sa (uint32, n) and bwt (uint8, n) may be given as the output buffers (for
        instance page-locked ones, which the device copies into directly)."""
        t = _as_text(text)
        n = len(t)
        if sa is None:
            sa = np.empty(max(n, 1), np.uint32)
        if bwt is None:
            bwt = np.empty(max(n, 1), np.uint8)
        if sa.dtype != np.uint32 or bwt.dtype != np.uint8 or len(sa) < n or len(bwt) < n:
            raise ValueError("sa must be uint32 and bwt uint8, each of at least n entries")
        out = bwt
        ticket = ctypes.c_uint64(0)
        _check(lib().sadcs_gpu_server_submit(self._handle, t.ctypes.data_as(_u8p), n, sa.ctypes.data_as(_u32p),
                                             out.ctypes.data_as(_u8p), ctypes.byref(ticket)))
        self._pending[ticket.value] = (t, sa, out, n)
        return int(ticket.value)

    def wait(self, ticket: int, timeout: float = -1.0):
        """Returns (sa, bwt, primary, latency (queued, device, total seconds), batch size)."""
        primary = ctypes.c_int64(0)
        latency = (ctypes.c_double * 3)()
        batch = ctypes.c_int32(0)
        status = lib().sadcs_gpu_server_wait(self._handle, int(ticket), float(timeout), ctypes.byref(primary),
                                             latency, ctypes.byref(batch))
        if status != GpuStatus.Ok and last_error() == "timed out":
            raise TimeoutError(f"request {ticket} still running")
        t, sa, out, n = self._pending.pop(ticket)
        _check(status)
        return sa[:n], out[:n], int(primary.value), tuple(latency), int(batch.value)

    def cancel(self, ticket: int) -> bool:
        """Cancels a request no worker has taken yet (True); its wait then raises GpuError
        ("cancelled"). False when it is being built, done, or unknown."""
        return lib().sadcs_gpu_server_cancel(self._handle, int(ticket)) == GpuStatus.Ok

    def fail_allocations(self, count: int) -> None:
        """Fault injection: the next `count` constructions fail their device allocation as an
        exhausted pool would; their requests raise GpuError (NotEnoughMemory)."""
        lib().sadcs_gpu_server_fail_allocations(self._handle, int(count))

    def counters(self):
        c, l = ctypes.c_int64(0), ctypes.c_int64(0)
        lib().sadcs_gpu_server_counters(self._handle, ctypes.byref(c), ctypes.byref(l))
        return int(c.value), int(l.value)

    def close(self) -> None:
        if getattr(self, "_handle", None):
            lib().sadcs_gpu_server_destroy(self._handle)
            self._handle = None
            self._pending.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
