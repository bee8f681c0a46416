"""sadcs_gpu_check_suffix_array_static, the suffix array check that allocates nothing, against
sadcs_gpu_check_suffix_array on the same device buffers: every verdict (ok, first failing index,
reason) must agree, on two calls in a row, so scratch left by one call cannot change the next one's
answer. This file sorts last so that it also runs after every other GPU test in one session."""
import numpy as np
import pytest

import oracle
import sadcs_b200 as sa
from sadcs_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _device(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _cases(text):
    good = oracle.naive_sa(text) if len(text) <= 20000 else oracle.doubling_sa(text)
    n = len(text)
    dup = good.copy()
    dup[n // 3] = dup[2 * n // 3]
    swap = good.copy()
    swap[n // 2], swap[n // 2 + 1] = swap[n // 2 + 1], swap[n // 2]
    far = good.copy()
    far[[5, n - 5]] = far[[n - 5, 5]]
    out = good.copy()
    out[n // 4] = n
    return {"correct": good, "duplicate entry": dup, "swapped neighbours": swap, "swapped far apart": far,
            "out of range": out}


def _memory_state():
    """What an allocation would change: the device's free memory, torch's allocator counters and the
    used and reserved bytes of the device's current stream-ordered memory pool."""
    import gc

    import torch

    gc.collect()  # tensors of earlier tests freed now, not between two readings
    torch.cuda.synchronize()
    state = {"free": torch.cuda.mem_get_info()[0], "torch_allocated": torch.cuda.memory_allocated(),
             "torch_reserved": torch.cuda.memory_reserved()}
    from cuda.bindings import runtime as rt

    error, device = rt.cudaGetDevice()
    assert error == rt.cudaError_t.cudaSuccess
    error, pool = rt.cudaDeviceGetMemPool(device)
    assert error == rt.cudaError_t.cudaSuccess
    for name in ("cudaMemPoolAttrUsedMemCurrent", "cudaMemPoolAttrReservedMemCurrent"):
        error, value = rt.cudaMemPoolGetAttribute(pool, getattr(rt.cudaMemPoolAttr, name))
        assert error == rt.cudaError_t.cudaSuccess
        state[name] = int(value)
    return state


def _compare(text):
    d_text = _device(text)
    for name, s in _cases(text).items():
        d_sa = _device(s.astype(np.uint32))
        expected = sa.check_suffix_array_device(d_text.data_ptr(), len(text), d_sa.data_ptr())
        for call in range(2):
            got = sa.check_suffix_array_static_device(d_text.data_ptr(), len(text), d_sa.data_ptr())
            assert got == expected, (name, call, got, expected)
        assert expected[0] == (name == "correct"), name


def test_matches_the_allocating_check_small():
    _compare(W.random_text(W.SplitMix(11), 5000, 4))


def test_matches_the_allocating_check_at_the_limit_then_small():
    # the largest accepted input, then a small one: the second call must not see the first's scratch
    _compare(W.natural_text(sa.STATIC_CHECK_MAX, seed=12))
    _compare(W.random_text(W.SplitMix(13), 777, 2))


def test_rejects_inputs_beyond_its_scratch():
    import torch

    n = sa.STATIC_CHECK_MAX + 1
    d_text = torch.zeros(n, dtype=torch.uint8, device="cuda")
    d_sa = torch.arange(n, dtype=torch.int32, device="cuda")
    with pytest.raises(sa.GpuError) as info:
        sa.check_suffix_array_static_device(d_text.data_ptr(), n, d_sa.data_ptr())
    assert "static scratch" in str(info.value)
    # the allocating entry point takes the same input
    ok, index, reason = sa.check_suffix_array_device(d_text.data_ptr(), n, d_sa.data_ptr())
    assert not ok


def test_a_call_allocates_nothing():
    """After one call (the first call on a device looks up the scratch array's address), further
    calls leave the device's free memory, torch's allocator and the stream-ordered pool unchanged."""
    text = W.natural_text(1 << 16, seed=14)
    d_text = _device(text)
    d_sa = _device(oracle.doubling_sa(text).astype(np.uint32))
    assert sa.check_suffix_array_static_device(d_text.data_ptr(), len(text), d_sa.data_ptr()) == (True, -1, None)
    before = _memory_state()
    for _ in range(2):
        assert sa.check_suffix_array_static_device(d_text.data_ptr(), len(text), d_sa.data_ptr()) == (True, -1, None)
    assert _memory_state() == before
