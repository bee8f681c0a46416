"""The C-ABI boundary without a GPU: libsadcs_gpu.so loads, exports every entry point that
include/*.h declares, and its host-side planning behaves (no kernel is launched here)."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

import oracle
import sadcs_b200 as sa

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "sadcs_gpu.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(sadcs_gpu_\w+)\s*\(", text)))


def test_header_declares_the_reference_surface():
    names = declared_functions()
    for required in ("sadcs_gpu_query_device", "sadcs_gpu_required_bytes", "sadcs_gpu_create_context",
                     "sadcs_gpu_destroy_context", "sadcs_gpu_suffix_array", "sadcs_gpu_bwt", "sadcs_gpu_rank_sample",
                     "sadcs_gpu_allocate_pinned", "sadcs_gpu_free_pinned", "sadcs_gpu_last_error",
                     "sadcs_gpu_sample_size", "sadcs_gpu_memory_reserve"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(sa.library_path()))
    missing = [name for name in declared_functions() if not hasattr(lib, name)]
    assert not missing, f"declared but not exported: {missing}"


def test_nm_shows_c_linkage():
    out = subprocess.run(["nm", "-D", "--defined-only", str(sa.library_path())], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (sadcs_gpu_\w+)", out))
    assert set(declared_functions()) <= exported


def test_sample_size_matches_the_oracle():
    for n in (0, 1, 2, 3, 31, 32, 33, 1000, 8 << 20, (1 << 31) - 1025, 3 << 30):
        assert sa.sample_size(n) == oracle.sample_size(n)


def test_required_bytes_plan():
    assert sa.required_bytes(0) == 0
    assert sa.required_bytes(-1) == -1
    assert sa.required_bytes(1 << 32) == -1
    previous = 0
    for n in (1, 1000, 1 << 20, 256 << 20, 3 << 30, (1 << 32) - 256):
        need = sa.required_bytes(n)
        assert need >= previous
        previous = need
    # SA + BWT from one construction: text, packed codes, ranks, lists, SA, BWT and small arrays;
    # from the carry threshold on, one word per input byte more for the carried code words.
    assert 10.0 < sa.required_bytes(64 << 20) / (64 << 20) < 11.5
    assert 18.0 < sa.required_bytes(3 << 30) / (3 << 30) < 19.5
    assert sa.memory_reserve() == 256 << 20


def test_calls_without_a_device_report_unavailable():
    pytest.importorskip("torch")
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(sa.GpuError) as err:
        sa.suffix_array(b"banana")
    assert err.value.status == sa.GpuStatus.Unavailable
    assert sa.last_error()
    with pytest.raises(sa.GpuError) as err:
        sa.Context(1000)
    assert err.value.status == sa.GpuStatus.Unavailable


def test_int32_api_refuses_texts_past_its_range():
    # Refused before any device work: the int32 suffix array cannot index 2 GiB - 1024 bytes and more.
    big = (1 << 31) - 1024
    status = sa.lib().sadcs_gpu_suffix_array(None, None, big, None, None)
    assert status == sa.GpuStatus.Failed
    assert "int32" in sa.last_error()
