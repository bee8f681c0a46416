"""The memory plan of a construction (sadcs_b200/csrc/sadcs_gpu.cu: planBatch, extentOf,
extentBound, planLayout), run as host code through tests/plan_harness.cu, which includes the
library source whole. A context allocates one slab for (capacity, texts) from extentBound; every
batch it admits is laid out from its own extent, and the construction refuses a layout larger than
the slab. So every field of a batch's extent, and its layout's peak with or without the SA and BWT
inside the slab, must stay within the bound's, for any texts of at most `capacity` bytes together
and at most `texts` of them. Also checked: texts start on a cover period, in order, with prefix-sum
sample and output bases, the residue classes partition the positions, and the merge's top level
fits one tile. CPU only."""
import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
SOURCE = HERE / "plan_harness.cu"
BUILT = HERE / "_build" / "libplan_harness.so"
CHECKS = {1: "planBatch refused", 2: "text not on a period", 3: "text length", 4: "texts out of order",
          5: "sample or output base", 6: "totals", 7: "span", 8: "class partition", 9: "top merge level over a tile",
          **{10 + f: f"extent field {name} over the bound" for f, name in enumerate(
              ["span", "slots", "live", "outputs", "largestClass", "splitterWords", "rows", "count"])},
          20: "layout peak over the bound's", 21: "layout peak over the context's slab"}
_lib = None


def harness():
    global _lib
    if _lib is None:
        sources = [SOURCE, *(ROOT / "sadcs_b200" / "csrc").glob("*"), ROOT / "include" / "sadcs_gpu.h"]
        newest = max(p.stat().st_mtime for p in sources)
        if not BUILT.exists() or BUILT.stat().st_mtime < newest:
            nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
            if not Path(nvcc).exists():
                pytest.skip("nvcc is needed to build the plan harness")
            BUILT.parent.mkdir(exist_ok=True)
            tmp = BUILT.with_suffix(".so.tmp")
            subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2", "-Xcompiler",
                            "-fPIC", "-shared", "-o", str(tmp), str(SOURCE)], check=True)
            tmp.replace(BUILT)
        L = ctypes.CDLL(str(BUILT))
        L.plan_check.restype = ctypes.c_int
        L.plan_check.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32,
                                 ctypes.POINTER(ctypes.c_int64)]
        L.plan_peak.restype = ctypes.c_uint64
        L.plan_peak.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.c_uint32]
        _lib = L
    return _lib


def check(lengths, capacity=None, texts=None):
    a = np.ascontiguousarray(lengths, dtype=np.uint64)
    capacity = int(a.sum()) if capacity is None else capacity
    texts = max(len(a), 1) if texts is None else texts
    detail = (ctypes.c_int64 * 3)()
    status = harness().plan_check(a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), len(a), capacity, texts, detail)
    assert status == 0, (CHECKS.get(status, status), list(detail), len(a), capacity, texts)


@pytest.mark.parametrize("n", [1, 2, 7, 31, 32, 33, 1000, 1467, 1468, 4096, 65535, 1 << 20, (1 << 20) + 13,
                               256 << 20, 3 << 30, (1 << 32) - 256])
def test_single_text_contexts(n):
    check([n])
    check([n], capacity=n + 1000)  # a context larger than the text


def test_random_batches_within_their_context():
    rng = np.random.default_rng(5)
    for _ in range(600):
        count = int(rng.integers(1, 300))
        lengths = np.exp(rng.uniform(0, np.log(1 << 22), count)).astype(np.uint64) + 1
        total = int(lengths.sum())
        check(lengths)  # the tightest context: exactly these bytes and texts
        check(lengths, capacity=total + int(rng.integers(0, 1 << 20)), texts=count + int(rng.integers(0, 50)))


def test_many_tiny_texts():
    # the per-text rounding to a period and the partial periods are the bound's slack terms
    for length in range(1, 70):
        check([length] * 5000)
    rng = np.random.default_rng(6)
    check(rng.integers(1, 40, 100_000))
    check(np.full(1 << 20, 1))  # the most texts a batch context takes


def test_batch_of_the_benchmark():
    from sadcs_b200 import workloads as W

    lengths = W.batch_lengths(4096, lo=1 << 10, hi=4 << 20, seed=4)
    check(lengths)
    peak = harness().plan_peak(np.ascontiguousarray(lengths, dtype=np.uint64).ctypes.data_as(
        ctypes.POINTER(ctypes.c_uint64)), len(lengths))
    assert 9 < peak / int(np.sum(lengths)) < 13  # about 10 bytes of device memory per input byte
