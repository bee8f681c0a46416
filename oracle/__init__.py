"""Test oracle for the suffix-array/BWT path. TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs may import this
package, and only as the checker (or, for the reference arm, as the timed CPU implementation).
The product package ``sadcs_b200`` never imports it.

Two libraries:

* ``liboracle.so`` - dcsa.c, a plain-C restatement of the reference's GPU path (cover mod 32 sample
  ranking, class derivation, difference-cover merge) plus an independent prefix-doubling SA, the BWT
  convention and 64-bit checkers. Built from committed source by ``make -C oracle``.
* ``_ref/libsadcs_ref.so`` - the reference's own CPU variant (src/cpu, src/common of acesds/sadcs),
  compiled from its sources by ``make -C oracle ref`` where they exist. Optional at run time: it is
  not committed (the sources are not ours) and is absent wherever it was not built.
* ``_ref/libsadcs_ref_gpu.so`` - the reference's own CUDA variant (src/cuda/gpusa.cu) for sm_100a,
  by ``make -C oracle ref-gpu``: the reference's GPU construction on the same device, for the
  timed comparison in bench.py and as a second parity source in the GPU tests.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libsadcs_ref.so"
REF_CLI = HERE / "_ref" / "sadcs_ref"
REF_GPU_SO = HERE / "_ref" / "libsadcs_ref_gpu.so"

_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)

_lib = None
_ref = None
_ref_gpu = None


def build(quiet: bool = True) -> None:
    """Compiles liboracle.so if it is missing or older than its source."""
    src = [HERE / "dcsa.c", HERE / "dcsa.h"]
    if ORACLE_SO.exists() and all(ORACLE_SO.stat().st_mtime >= s.stat().st_mtime for s in src):
        return
    subprocess.run(["make", "-C", str(HERE), "liboracle.so"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(ORACLE_SO))
        L.oracle_sample_size.restype = ctypes.c_int64
        L.oracle_sample_size.argtypes = [ctypes.c_int64]
        for name in ("oracle_naive_sa", "oracle_doubling_sa", "oracle_dc_sa", "oracle_dc_sample_ranks"):
            f = getattr(L, name)
            f.restype = ctypes.c_int
            f.argtypes = [_u8p, ctypes.c_int64, _u32p]
        L.oracle_dc_class_lists.restype = ctypes.c_int
        L.oracle_dc_class_lists.argtypes = [_u8p, ctypes.c_int64, _u32p, _u32p, _i64p]
        L.oracle_dc_merge.restype = ctypes.c_int
        L.oracle_dc_merge.argtypes = [_u8p, ctypes.c_int64, _u32p, _u32p, _i64p, _u32p]
        L.oracle_sample_ranks_from_sa.restype = None
        L.oracle_sample_ranks_from_sa.argtypes = [_u32p, ctypes.c_int64, _u32p]
        L.oracle_bwt_from_sa.restype = ctypes.c_int64
        L.oracle_bwt_from_sa.argtypes = [_u8p, ctypes.c_int64, _u32p, _u8p]
        L.oracle_check_sa.restype = ctypes.c_int
        L.oracle_check_sa.argtypes = [_u8p, ctypes.c_int64, _u32p, _i64p]
        L.oracle_check_bwt.restype = ctypes.c_int
        L.oracle_check_bwt.argtypes = [_u8p, ctypes.c_int64, _u8p, ctypes.c_int64, _i64p]
        L.oracle_lcp.restype = ctypes.c_int
        L.oracle_lcp.argtypes = [_u8p, ctypes.c_int64, _u32p, _u32p]
        L.oracle_cover_tables.restype = None
        L.oracle_cover_tables.argtypes = [_u8p, _u8p, _u8p]
        _lib = L
    return _lib


def ref_available() -> bool:
    return REF_SO.exists()


def ref() -> ctypes.CDLL:
    """The reference's own CPU build; raises if it was not built."""
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} not built (make -C oracle ref, needs the reference sources)")
        L = ctypes.CDLL(str(REF_SO))
        L.ref_build_sa.restype = ctypes.c_int
        L.ref_build_sa.argtypes = [_u8p, ctypes.c_int32, _i32p, ctypes.c_int]
        L.ref_build_sa_padded.restype = ctypes.c_int
        L.ref_build_sa_padded.argtypes = [_u8p, ctypes.c_int32, _i32p, ctypes.c_int]
        L.ref_build_bwt.restype = ctypes.c_int32
        L.ref_build_bwt.argtypes = [_u8p, ctypes.c_int32, _u8p, ctypes.c_int]
        L.ref_build_bwt_padded.restype = ctypes.c_int32
        L.ref_build_bwt_padded.argtypes = [_u8p, ctypes.c_int32, _u8p, _i32p, ctypes.c_int]
        L.ref_check_sa.restype = ctypes.c_int
        L.ref_check_sa.argtypes = [_u8p, ctypes.c_int32, _i32p, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]
        L.ref_check_bwt.restype = ctypes.c_int
        L.ref_check_bwt.argtypes = [_u8p, ctypes.c_int32, _u8p, ctypes.c_int32, ctypes.POINTER(ctypes.c_longlong)]
        L.ref_set_threads.restype = None
        L.ref_set_threads.argtypes = [ctypes.c_int]
        L.ref_max_threads.restype = ctypes.c_int
        L.ref_text_padding.restype = ctypes.c_int
        L.ref_max_text_size.restype = ctypes.c_longlong
        _ref = L
    return _ref


def ref_gpu_available() -> bool:
    return REF_GPU_SO.exists()


def ref_gpu() -> ctypes.CDLL:
    """The reference's own CUDA build; raises if it was not built."""
    global _ref_gpu
    if _ref_gpu is None:
        if not REF_GPU_SO.exists():
            raise FileNotFoundError(f"{REF_GPU_SO} not built (make -C oracle ref-gpu, needs the reference sources)")
        L = ctypes.CDLL(str(REF_GPU_SO))
        L.ref_gpu_create_context.restype = ctypes.c_int
        L.ref_gpu_create_context.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]
        L.ref_gpu_destroy_context.restype = None
        L.ref_gpu_destroy_context.argtypes = [ctypes.c_void_p]
        L.ref_gpu_suffix_array.restype = ctypes.c_int
        L.ref_gpu_suffix_array.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_int32, _i32p,
                                           ctypes.POINTER(ctypes.c_double)]
        L.ref_gpu_bwt.restype = ctypes.c_int
        L.ref_gpu_bwt.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_int32, _u8p, _i32p, ctypes.POINTER(ctypes.c_double)]
        L.ref_gpu_allocate_pinned.restype = ctypes.c_void_p
        L.ref_gpu_allocate_pinned.argtypes = [ctypes.c_size_t]
        L.ref_gpu_free_pinned.restype = None
        L.ref_gpu_free_pinned.argtypes = [ctypes.c_void_p]
        L.ref_gpu_last_error.restype = ctypes.c_char_p
        _ref_gpu = L
    return _ref_gpu


class RefGpuContext:
    """A context of the reference's CUDA build (gpuCreateContext) for texts of up to capacity bytes."""

    def __init__(self, capacity: int):
        L = ref_gpu()
        self.handle = ctypes.c_void_p()
        status = L.ref_gpu_create_context(int(capacity), ctypes.byref(self.handle))
        if status != 0:
            raise RuntimeError(f"reference gpuCreateContext: status {status}: {L.ref_gpu_last_error().decode()}")

    def suffix_array(self, text: np.ndarray, out: np.ndarray | None = None) -> tuple[np.ndarray, float]:
        """(SA, device seconds) of the reference's GPU construction."""
        L = ref_gpu()
        t = _text(text)
        n = len(t)
        sa = out if out is not None else np.zeros(max(n, 1), np.int32)
        seconds = ctypes.c_double(0)
        status = L.ref_gpu_suffix_array(self.handle, _ptr(_nonempty(t), _u8p), n, _ptr(sa, _i32p),
                                        ctypes.byref(seconds))
        if status != 0:
            raise RuntimeError(f"reference gpuSuffixArray: status {status}: {L.ref_gpu_last_error().decode()}")
        return sa[:n], seconds.value

    def bwt(self, text: np.ndarray, out: np.ndarray | None = None) -> tuple[np.ndarray, int, float]:
        """(BWT, primary, device seconds) of the reference's GPU construction."""
        L = ref_gpu()
        t = _text(text)
        n = len(t)
        bwt = out if out is not None else np.zeros(max(n, 1), np.uint8)
        primary = ctypes.c_int32(0)
        seconds = ctypes.c_double(0)
        status = L.ref_gpu_bwt(self.handle, _ptr(_nonempty(t), _u8p), n, _ptr(bwt, _u8p), ctypes.byref(primary),
                               ctypes.byref(seconds))
        if status != 0:
            raise RuntimeError(f"reference gpuBwt: status {status}: {L.ref_gpu_last_error().decode()}")
        return bwt[:n], int(primary.value), seconds.value

    def close(self) -> None:
        if self.handle:
            ref_gpu().ref_gpu_destroy_context(self.handle)
            self.handle = ctypes.c_void_p()


def ref_gpu_pinned(nbytes: int) -> np.ndarray | None:
    """Page-locked host memory from the reference's gpuAllocatePinned (None if unavailable); free
    with ref_gpu_free_pinned."""
    p = ref_gpu().ref_gpu_allocate_pinned(int(nbytes))
    if not p:
        return None
    return np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_uint8)), shape=(int(nbytes),))


def ref_gpu_free_pinned(a: np.ndarray) -> None:
    ref_gpu().ref_gpu_free_pinned(ctypes.c_void_p(a.ctypes.data))


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _text(text) -> np.ndarray:
    a = np.frombuffer(bytes(text), dtype=np.uint8) if isinstance(text, (bytes, bytearray)) else np.asarray(text)
    a = np.ascontiguousarray(a, dtype=np.uint8)
    # Keep a non-empty buffer so ctypes gets a valid pointer for n == 0.
    return a if a.size else np.zeros(1, dtype=np.uint8)[:0].copy()


def _nonempty(a: np.ndarray) -> np.ndarray:
    return a if a.size else np.zeros(1, dtype=a.dtype)


# ---- the restatement -------------------------------------------------------------------------

def sample_size(n: int) -> int:
    return int(lib().oracle_sample_size(n))


def cover_tables():
    below = np.zeros(32, np.uint8)
    tie = np.zeros(32 * 32, np.uint8)
    cls = np.zeros(32, np.uint8)
    lib().oracle_cover_tables(_ptr(below, _u8p), _ptr(tie, _u8p), _ptr(cls, _u8p))
    return below, tie.reshape(32, 32), cls


def _sa_with(fn, text) -> np.ndarray:
    t = _nonempty(_text(text))
    n = len(_text(text))
    sa = np.zeros(max(n, 1), np.uint32)
    rc = fn(_ptr(t, _u8p), n, _ptr(sa, _u32p))
    if rc != 0:
        raise RuntimeError(f"oracle failed ({rc})")
    return sa[:n]


def naive_sa(text) -> np.ndarray:
    return _sa_with(lib().oracle_naive_sa, text)


def doubling_sa(text) -> np.ndarray:
    return _sa_with(lib().oracle_doubling_sa, text)


def dc_sa(text) -> np.ndarray:
    return _sa_with(lib().oracle_dc_sa, text)


def dc_sample_ranks(text) -> np.ndarray:
    t = _text(text)
    n = len(t)
    ranks = np.zeros(sample_size(n) + 1, np.uint32)
    rc = lib().oracle_dc_sample_ranks(_ptr(_nonempty(t), _u8p), n, _ptr(ranks, _u32p))
    if rc != 0:
        raise RuntimeError(f"oracle failed ({rc})")
    return ranks[: sample_size(n)]


def dc_class_lists(text, ranks: np.ndarray):
    t = _text(text)
    n = len(t)
    r = np.ascontiguousarray(np.concatenate([ranks.astype(np.uint32), np.zeros(1, np.uint32)]))
    lists = np.zeros(max(n, 1), np.uint32)
    start = np.zeros(8, np.int64)
    rc = lib().oracle_dc_class_lists(_ptr(_nonempty(t), _u8p), n, _ptr(r, _u32p), _ptr(lists, _u32p),
                                     _ptr(start, _i64p))
    if rc != 0:
        raise RuntimeError(f"oracle failed ({rc})")
    return lists[:n], start


def sample_ranks_from_sa(sa: np.ndarray, n: int) -> np.ndarray:
    sa = np.ascontiguousarray(sa, dtype=np.uint32)
    ranks = np.zeros(sample_size(n) + 1, np.uint32)
    lib().oracle_sample_ranks_from_sa(_ptr(_nonempty(sa), _u32p), n, _ptr(ranks, _u32p))
    return ranks[: sample_size(n)]


def class_lists_from_sa(sa: np.ndarray, n: int):
    """Each class list is the suffix array restricted to that class (every list is sorted)."""
    _, _, cls = cover_tables()
    sa = np.asarray(sa, dtype=np.uint32)
    c = cls[sa % 32]
    parts = [sa[c == d] for d in range(7)]
    start = np.zeros(8, np.int64)
    start[1:] = np.cumsum([len(p) for p in parts])
    return (np.concatenate(parts) if n else np.zeros(0, np.uint32)), start


def bwt_from_sa(text, sa: np.ndarray):
    t = _text(text)
    n = len(t)
    sa = np.ascontiguousarray(sa, dtype=np.uint32)
    bwt = np.zeros(max(n, 1), np.uint8)
    primary = lib().oracle_bwt_from_sa(_ptr(_nonempty(t), _u8p), n, _ptr(_nonempty(sa), _u32p), _ptr(bwt, _u8p))
    return bwt[:n], int(primary)


def lcp(text, sa: np.ndarray) -> np.ndarray:
    """lcp[0] = 0, lcp[r] = common prefix length of suffixes sa[r - 1] and sa[r] (uint32)."""
    t = _text(text)
    n = len(t)
    sa = np.ascontiguousarray(sa, dtype=np.uint32)
    out = np.zeros(max(n, 1), np.uint32)
    if not lib().oracle_lcp(_ptr(_nonempty(t), _u8p), n, _ptr(_nonempty(sa), _u32p), _ptr(out, _u32p)):
        raise MemoryError("oracle_lcp")
    return out[:n]


def check_sa(text, sa: np.ndarray):
    t = _text(text)
    n = len(t)
    sa = np.ascontiguousarray(sa, dtype=np.uint32)
    idx = ctypes.c_int64(-1)
    ok = lib().oracle_check_sa(_ptr(_nonempty(t), _u8p), n, _ptr(_nonempty(sa), _u32p), ctypes.byref(idx))
    return bool(ok), int(idx.value)


def check_bwt(text, bwt: np.ndarray, primary: int):
    t = _text(text)
    n = len(t)
    bwt = np.ascontiguousarray(bwt, dtype=np.uint8)
    idx = ctypes.c_int64(-1)
    ok = lib().oracle_check_bwt(_ptr(_nonempty(t), _u8p), n, _ptr(_nonempty(bwt), _u8p), int(primary),
                                ctypes.byref(idx))
    return bool(ok), int(idx.value)


# ---- the reference's own CPU build -----------------------------------------------------------

def ref_sa(text, cover: int = 128, threads: int | None = None) -> np.ndarray:
    L = ref()
    if threads:
        L.ref_set_threads(int(threads))
    t = _text(text)
    n = len(t)
    sa = np.zeros(max(n, 1), np.int32)
    if not L.ref_build_sa(_ptr(_nonempty(t), _u8p), n, _ptr(sa, _i32p), cover):
        raise RuntimeError("reference buildSuffixArray refused")
    return sa[:n]


def ref_bwt(text, cover: int = 128, threads: int | None = None):
    L = ref()
    if threads:
        L.ref_set_threads(int(threads))
    t = _text(text)
    n = len(t)
    bwt = np.zeros(max(n, 1), np.uint8)
    primary = L.ref_build_bwt(_ptr(_nonempty(t), _u8p), n, _ptr(bwt, _u8p), cover)
    if primary < 0:
        raise RuntimeError("reference buildBwt refused")
    return bwt[:n], int(primary)


def ref_check_sa(text, sa: np.ndarray, mode: int = 0):
    L = ref()
    t = _text(text)
    n = len(t)
    sa = np.ascontiguousarray(sa, dtype=np.int32)
    idx = ctypes.c_longlong(-1)
    ok = L.ref_check_sa(_ptr(_nonempty(t), _u8p), n, _ptr(_nonempty(sa), _i32p), mode, ctypes.byref(idx))
    return bool(ok), int(idx.value)


def ref_check_bwt(text, bwt: np.ndarray, primary: int):
    L = ref()
    t = _text(text)
    n = len(t)
    bwt = np.ascontiguousarray(bwt, dtype=np.uint8)
    idx = ctypes.c_longlong(-1)
    ok = L.ref_check_bwt(_ptr(_nonempty(t), _u8p), n, _ptr(_nonempty(bwt), _u8p), int(primary), ctypes.byref(idx))
    return bool(ok), int(idx.value)


def host_cores() -> int:
    return len(os.sched_getaffinity(0))
