"""The LCP array of a suffix array (sadcs_gpu_lcp, sadcs_b200/csrc/lcp.cuh) against the oracle's
Kasai LCP (oracle_lcp, pinned in test_oracle.py by direct comparison of neighbouring suffixes).

CPU tests run the kernels' own per-thread bodies as host code (tests/lcp_emulation.cu, built with
nvcc): every pass in launch order, the warp pass as a minimum over 32 emulated lanes, each text
read checked against the text's end. They cover the word-load and the byte-load paths, the hand-
over to the warp pass, an output that is the suffix array itself, and corrupted suffix arrays
(results unspecified, reads still inside the text). GPU tests call the C ABI on device buffers.
The reference computes no LCP array, so there is no reference output to pin against."""
import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
import sadcs_b200 as sa
from sadcs_b200 import workloads as W
from tests.golden.make_golden import small_inputs

HERE = Path(__file__).resolve().parent
SOURCE = HERE / "lcp_emulation.cu"
HEADERS = [HERE.parent / "sadcs_b200" / "csrc" / name for name in ("lcp.cuh", "common.cuh", "primitives.cuh")]
BUILT = HERE / "_build" / "liblcp_emulation.so"

_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_emulation = None


def emulation():
    global _emulation
    if _emulation is None:
        newest = max(p.stat().st_mtime for p in [SOURCE, *HEADERS])
        if not BUILT.exists() or BUILT.stat().st_mtime < newest:
            nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
            if not Path(nvcc).exists():
                pytest.skip("nvcc is needed to build the host emulation of the LCP kernels")
            BUILT.parent.mkdir(exist_ok=True)
            tmp = BUILT.with_suffix(".so.tmp")
            subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2", "-Xcompiler",
                            "-fPIC", "-shared", "-o", str(tmp), str(SOURCE)], check=True)
            tmp.replace(BUILT)
        L = ctypes.CDLL(str(BUILT))
        L.lcp_emulate.restype = ctypes.c_int
        L.lcp_emulate.argtypes = [_u8p, ctypes.c_int64, _u32p, _u32p, ctypes.c_int, ctypes.c_uint32, _i64p, _i64p]
        _emulation = L
    return _emulation


def emulate(text, suffixes, aligned=True, fill=0xA5A5A5A5, out=None):
    """(lcp, end of the first read past the text or 0, comparisons handed to the warp pass)."""
    t = np.ascontiguousarray(text, dtype=np.uint8)
    s = np.ascontiguousarray(suffixes, dtype=np.uint32)
    if out is None:
        out = np.zeros(len(t), np.uint32)
    bad, unfinished = ctypes.c_int64(), ctypes.c_int64()
    keep = [t if len(t) else np.zeros(1, np.uint8), s if len(s) else np.zeros(1, np.uint32),
            out if len(out) else np.zeros(1, np.uint32)]
    emulation().lcp_emulate(keep[0].ctypes.data_as(_u8p), len(t), keep[1].ctypes.data_as(_u32p),
                            keep[2].ctypes.data_as(_u32p), int(aligned), fill, ctypes.byref(bad),
                            ctypes.byref(unfinished))
    return out, bad.value, unfinished.value


def suffix_array(text):
    return oracle.doubling_sa(text) if len(text) else np.zeros(0, np.uint32)


def expected_lcp(text, s):
    return oracle.lcp(text, s) if len(text) else np.zeros(0, np.uint32)


def cases():
    rng = W.SplitMix(31)
    out = [(name, t) for name, t in small_inputs()]
    out += [("runs 5000", W.run_text(5000)),
            ("run with one break", np.concatenate([W.run_text(3000), [ord("b")], W.run_text(2999)]).astype(np.uint8)),
            ("period 3 x 4000", W.periodic_text(rng, 12000, 3)),
            ("fibonacci 20000", W.fibonacci_text(20000)),
            ("thue-morse 16384", W.thue_morse_text(16384)),
            ("random sigma=4 30000", W.random_text(rng, 30000, 4)),
            ("natural 200000", W.natural_text(200_000, seed=5)),
            ("genome 300000", W.genome_text(300_000, seed=6, segment=8192))]
    return out


CASES = cases()


@pytest.mark.parametrize("aligned", [True, False], ids=["word loads", "byte loads"])
@pytest.mark.parametrize("name,text", CASES, ids=[c[0] for c in CASES])
def test_emulated_kernels_match_the_oracle(name, text, aligned):
    s = suffix_array(text)
    got, bad, _ = emulate(text, s, aligned)
    assert bad == 0, f"a text read ends at {bad}, past n = {len(text)}"
    assert np.array_equal(got, expected_lcp(text, s))


def test_long_common_prefixes_reach_the_warp_pass():
    # A run's whole LCP array comes from one irreducible comparison of n - 1 characters, which the
    # first thread hands over after 256; the genome-like copies hand over many shorter ones.
    for text, least in ((W.run_text(100_000), 1), (W.genome_text(300_000, seed=6, segment=8192), 10)):
        s = suffix_array(text)
        got, bad, unfinished = emulate(text, s)
        assert bad == 0 and unfinished >= least
        assert np.array_equal(got, expected_lcp(text, s))


def test_output_may_be_the_suffix_array_itself():
    text = W.natural_text(50_000, seed=8)
    s = suffix_array(text)
    expected = expected_lcp(text, s)
    inplace = s.copy()
    got, bad, _ = emulate(text, inplace, out=inplace)
    assert got is inplace and bad == 0
    assert np.array_equal(inplace, expected)


@pytest.mark.parametrize("fill", [0xA5A5A5A5, 0, 7, 0xFFFFFFFF])
def test_corrupt_suffix_arrays_read_only_inside_the_text(fill):
    text = W.genome_text(20_000, seed=9, segment=2048)
    n = len(text)
    good = suffix_array(text)
    dup = good.copy()
    dup[100:200] = dup[0]
    big = good.copy()
    big[::7] = n + 5
    shuffled = good.copy()
    np.random.default_rng(1).shuffle(shuffled)
    for s in (dup, big, shuffled, np.full(n, 0xFFFFFFFF, np.uint32)):
        _, bad, _ = emulate(text, s, fill=fill)
        assert bad == 0
        _, bad, _ = emulate(text, s, aligned=False, fill=fill)
        assert bad == 0


# ---- on the device, through the C ABI -------------------------------------------------------------


def _device(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _device_lcp(text, s, offset=0, inplace=False):
    import torch

    n = len(text)
    if offset:
        backing = torch.zeros(n + offset, dtype=torch.uint8, device="cuda")
        backing[offset:] = _device(text)
        d_text = backing[offset:]
        assert d_text.data_ptr() % 8 == offset % 8
    else:
        d_text = _device(text)
    d_sa = _device(s.astype(np.uint32).view(np.int32))
    d_out = d_sa if inplace else torch.empty(n, dtype=torch.int32, device="cuda")
    sa.lcp_device(d_text.data_ptr(), n, d_sa.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    return d_out.cpu().numpy().view(np.uint32)


@pytest.mark.gpu
@pytest.mark.parametrize("name,text", CASES, ids=[c[0] for c in CASES])
def test_device_matches_the_oracle(name, text):
    s = suffix_array(text)
    assert np.array_equal(_device_lcp(text, s), expected_lcp(text, s))


@pytest.mark.gpu
def test_device_unaligned_text_and_in_place():
    text = W.genome_text(100_000, seed=10, segment=4096)
    s = suffix_array(text)
    expected = expected_lcp(text, s)
    for offset in (1, 3, 5):
        assert np.array_equal(_device_lcp(text, s, offset=offset), expected)
    assert np.array_equal(_device_lcp(text, s, inplace=True), expected)


@pytest.mark.gpu
@pytest.mark.parametrize("make", [lambda: W.natural_text(8 << 20, seed=2),
                                  lambda: W.genome_text(16 << 20, seed=3, segment=1 << 18),
                                  lambda: W.run_text(1 << 20)],
                         ids=["natural 8 MiB", "genome-like 16 MiB", "run 1 MiB"])
def test_device_large_texts_with_the_library_suffix_array(make):
    text = make()
    suffixes, _, _ = sa.build(text)
    assert np.array_equal(_device_lcp(text, suffixes), oracle.lcp(text, suffixes))


@pytest.mark.gpu
def test_device_empty_and_single():
    import torch

    sa.lcp_device(0, 0, 0, 0)
    one = torch.tensor([65], dtype=torch.uint8, device="cuda")
    s = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.full((1,), 9, dtype=torch.int32, device="cuda")
    sa.lcp_device(one.data_ptr(), 1, s.data_ptr(), out.data_ptr())
    assert out.item() == 0
