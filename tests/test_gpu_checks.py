"""Device-side checkers and the inverse BWT: they accept what the oracle accepts and catch the
reference selftest's planted errors (src/cli/selftest.cpp:309-385)."""
import numpy as np
import pytest

import oracle
import sadcs_b200 as sa
from sadcs_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _device(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_suffix_array_check_accepts_and_rejects():
    rng = W.SplitMix(7)
    text = W.random_text(rng, 3000, 3)
    good = oracle.naive_sa(text)
    d_text = _device(text)
    d_good = _device(good)  # held until the check returns: a freed block could be handed out again
    ok, index, _ = sa.check_suffix_array_device(d_text.data_ptr(), len(text), d_good.data_ptr())
    assert ok and index == -1
    mutations = {
        "swapped neighbours": lambda s: s.__setitem__(slice(1000, 1002), s[1000:1002][::-1].copy()),
        "swapped far apart": lambda s: s.__setitem__([10, 2900], s[[2900, 10]]),
        "duplicate entry": lambda s: s.__setitem__(500, s[1500]),
        "out of range": lambda s: s.__setitem__(42, len(s)),
    }
    for name, mutate in mutations.items():
        bad = good.copy()
        mutate(bad)
        d_bad = _device(bad)
        ok, index, reason = sa.check_suffix_array_device(d_text.data_ptr(), len(text), d_bad.data_ptr())
        assert not ok and index >= 0 and reason, name
        if name == "duplicate entry":
            # the smallest index of any repeated entry, whatever order the scatter ran in
            assert (index, reason) == (500, "duplicate entry")


def test_bwt_check_and_inverse():
    import torch

    for text in (W.natural_text(1 << 20, seed=3), W.run_text(5000), W.fibonacci_text(9000),
                 np.frombuffer(b"mississippi", np.uint8), W.random_text(W.SplitMix(2), 70000, 256)):
        expected = oracle.doubling_sa(text)
        bwt, primary = oracle.bwt_from_sa(text, expected)
        d_text, d_bwt = _device(text), _device(bwt)
        ok, index = sa.check_bwt_device(d_text.data_ptr(), len(text), d_bwt.data_ptr(), primary)
        assert ok and index == -1
        out = torch.zeros(len(text), dtype=torch.uint8, device="cuda")
        sa.inverse_bwt_device(d_bwt.data_ptr(), len(text), primary, out.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), text)
    text = W.random_text(W.SplitMix(7), 3000, 3)
    bwt, primary = oracle.bwt_from_sa(text, oracle.naive_sa(text))
    changed = bwt.copy()
    changed[1234] ^= 1
    d_text = _device(text)
    for name, b, p in (("changed character", changed, primary),
                       ("primary off by one", bwt, primary + 1 if primary < 3000 else primary - 1),
                       ("primary 0", bwt, 0)):
        d_b = _device(b)
        ok, _ = sa.check_bwt_device(d_text.data_ptr(), len(text), d_b.data_ptr(), p)
        assert not ok, name


def test_inverse_bwt_across_chunks_past_2g():
    """Past 2^29 positions the inverse's stable byte pass runs as chunks with carried digit bases,
    and past 2^31 its scratch offsets pass 2^32 words: a 2 GiB + 4 KiB text over {A,C,G,T} (five
    chunks) built by this library must come back exactly, and one changed byte must be caught."""
    import torch

    n = (1 << 31) + 4099
    g = torch.Generator(device="cuda").manual_seed(21)
    d_text = torch.randint(0, 4, (n,), dtype=torch.uint8, device="cuda", generator=g)
    d_text.mul_(2).add_(65)  # A C E G: four symbols, code order = byte order
    d_sa = torch.empty(n, dtype=torch.int32, device="cuda")
    d_bwt = torch.empty(n, dtype=torch.uint8, device="cuda")
    ctx = sa.Context(n)
    primary = sa.build_device(d_text.data_ptr(), n, d_sa.data_ptr(), d_bwt.data_ptr(), context=ctx)
    ctx.close()
    ok, where, _ = sa.check_suffix_array_device(d_text.data_ptr(), n, d_sa.data_ptr())
    assert ok, where
    del d_sa
    torch.cuda.empty_cache()
    out = torch.zeros(n, dtype=torch.uint8, device="cuda")
    sa.inverse_bwt_device(d_bwt.data_ptr(), n, primary, out.data_ptr())
    torch.cuda.synchronize()
    assert torch.equal(out, d_text)
    del out
    torch.cuda.empty_cache()
    ok, where = sa.check_bwt_device(d_text.data_ptr(), n, d_bwt.data_ptr(), primary)
    assert ok, where
    d_bwt[n - 7] ^= 2  # one changed byte in the last chunk
    ok, _ = sa.check_bwt_device(d_text.data_ptr(), n, d_bwt.data_ptr(), primary)
    assert not ok


def test_host_buffer_checks_agree_with_the_device_checks():
    """sadcs_gpu_check_suffix_array_host / sadcs_gpu_check_bwt_host (checkSuffixArray and checkBwt
    with host buffers) give the verdicts of the device-buffer entry points."""
    text = W.natural_text(1 << 18, seed=31)
    good = oracle.doubling_sa(text).astype(np.uint32)
    bwt, primary = oracle.bwt_from_sa(text, good)
    assert sa.check_suffix_array(text, good) == (True, -1, None)
    assert sa.check_bwt(text, bwt, primary) == (True, -1)
    d_text = _device(text)
    for name, mutate in (("swap", lambda s: s.__setitem__([7, 8], s[[8, 7]])),
                         ("duplicate", lambda s: s.__setitem__(100, s[5000])),
                         ("out of range", lambda s: s.__setitem__(3, len(s) + 3))):
        bad = good.copy()
        mutate(bad)
        d_bad = _device(bad)
        expected = sa.check_suffix_array_device(d_text.data_ptr(), len(text), d_bad.data_ptr())
        assert sa.check_suffix_array(text, bad) == expected and not expected[0], name
    changed = bwt.copy()
    changed[len(text) // 2] ^= 0x20
    d_changed = _device(changed)
    expected = sa.check_bwt_device(d_text.data_ptr(), len(text), d_changed.data_ptr(), primary)
    assert sa.check_bwt(text, changed, primary) == expected and not expected[0]
    assert sa.check_bwt(text, bwt, 0) == (False, 0)
    assert sa.check_bwt(text[:0], bwt[:0], 0) == (True, -1)
