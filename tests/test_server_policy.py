"""The serving loop's grouping and admission policy (sadcs_b200/csrc/server_policy.h, the code the
server's workers run) built as host code and checked against its stated rules: arrival order, a
large head alone, small requests together up to the batch's bytes and texts, and admission by
device footprint beside the running constructions. CPU only."""
import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
SOURCE = HERE / "server_policy_harness.cpp"
HEADER = HERE.parent / "sadcs_b200" / "csrc" / "server_policy.h"
BUILT = HERE / "_build" / "libserver_policy.so"
_lib = None


def policy():
    global _lib
    if _lib is None:
        newest = max(SOURCE.stat().st_mtime, HEADER.stat().st_mtime)
        if not BUILT.exists() or BUILT.stat().st_mtime < newest:
            cxx = shutil.which("g++")
            if not cxx:
                pytest.skip("g++ is needed to build the policy harness")
            BUILT.parent.mkdir(exist_ok=True)
            tmp = BUILT.with_suffix(".so.tmp")
            subprocess.run([cxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-o", str(tmp), str(SOURCE)], check=True)
            tmp.replace(BUILT)
        L = ctypes.CDLL(str(BUILT))
        L.policy_group_size.restype = ctypes.c_size_t
        L.policy_group_size.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.c_size_t, ctypes.c_uint64,
                                        ctypes.c_uint64, ctypes.c_uint32]
        L.policy_admits.restype = ctypes.c_int
        L.policy_admits.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]
        _lib = L
    return _lib


def group_size(lengths, small_limit, batch_bytes, batch_texts):
    a = np.ascontiguousarray(lengths, dtype=np.uint64)
    keep = a if len(a) else np.zeros(1, np.uint64)
    return policy().policy_group_size(keep.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), len(a), small_limit,
                                      batch_bytes, batch_texts)


def stated_rule(lengths, small_limit, batch_bytes, batch_texts):
    """The grouping rule as documented, restated directly."""
    if not lengths:
        return 0
    if lengths[0] > small_limit:
        return 1
    take, total = 1, lengths[0]
    for n in lengths[1:]:
        if n > small_limit or total + n > batch_bytes or take >= batch_texts:
            break
        take, total = take + 1, total + n
    return take


def test_grouping_cases():
    kib = 1 << 10
    assert group_size([], 64 * kib, 1 << 20, 8) == 0
    assert group_size([1 << 30, 10, 10], 64 * kib, 1 << 20, 8) == 1  # a large head goes alone
    assert group_size([10, 1 << 30, 10], 64 * kib, 1 << 20, 8) == 1  # a large one ends the group
    assert group_size([10] * 20, 64 * kib, 1 << 20, 8) == 8  # at most batch_texts
    assert group_size([60 * kib] * 20, 64 * kib, 200 * kib, 64) == 3  # at most batch_bytes
    assert group_size([64 * kib, 64 * kib], 64 * kib, 128 * kib, 64) == 2  # limits are inclusive
    assert group_size([64 * kib + 1], 64 * kib, 1 << 20, 64) == 1


def test_grouping_matches_the_stated_rule_on_random_queues():
    rng = np.random.default_rng(3)
    for _ in range(2000):
        count = int(rng.integers(0, 40))
        lengths = [int(x) for x in np.exp(rng.uniform(0, np.log(1 << 26), count)).astype(np.uint64)]
        small = int(rng.choice([1 << 12, 1 << 16, 1 << 20]))
        batch = small * int(rng.integers(1, 64))
        texts = int(rng.integers(1, 32))
        got = group_size(lengths, small, batch, texts)
        assert got == stated_rule(lengths, small, batch, texts), (lengths, small, batch, texts)
        if count:
            assert sum(lengths[:got]) <= batch or got == 1


def test_admission():
    admits = policy().policy_admits
    assert admits(10, 0, 5)  # alone on an idle device: always
    assert admits(10, 0, 0)
    assert admits(5, 5, 10)  # fits beside the running ones (inclusive)
    assert not admits(6, 5, 10)
    assert not admits(1, 10, 10)


def test_small_lane_starts_at_the_first_small_request():
    """Worker 0 of two or more is the small lane: its group starts at the first small request of the
    queue (large ones ahead of it are left to the other workers); the others start at the head."""
    L = policy()
    L.policy_group_start.restype = ctypes.c_size_t
    L.policy_group_start.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.c_size_t, ctypes.c_uint64, ctypes.c_int]

    def start(lengths, small_limit, lane):
        a = np.ascontiguousarray(lengths, dtype=np.uint64)
        keep = a if len(a) else np.zeros(1, np.uint64)
        return L.policy_group_start(keep.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), len(a), small_limit, lane)

    assert start([5000, 6000, 10, 20], 100, 1) == 2
    assert start([5000, 6000, 10, 20], 100, 0) == 0
    assert start([5000, 6000], 100, 1) == 2  # nothing small: the lane waits
    assert start([], 100, 1) == 0
    assert start([10, 5000], 100, 1) == 0
    assert [L.policy_is_small_lane(w, n) for n in (1, 2, 3) for w in range(n)] == [0, 1, 0, 1, 0, 0]
    rng = np.random.default_rng(9)
    for _ in range(500):
        lengths = [int(x) for x in rng.choice([10, 50, 90, 1000, 5000], size=int(rng.integers(0, 12)))]
        got = start(lengths, 100, 1)
        expected = next((k for k, n in enumerate(lengths) if n <= 100), len(lengths))
        assert got == expected
        # the lane's group is the grouping rule applied from there on
        if got < len(lengths):
            assert group_size(lengths[got:], 100, 400, 3) == stated_rule(lengths[got:], 100, 400, 3)
