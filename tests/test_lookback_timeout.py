"""Failure detection of the radix passes' bounded wait, without a GPU fault: one pass whose only
block waits on a predecessor's status that nothing ever publishes (sadcs_gpu_test_lookback_timeout).
With a short limit the block must give up on its own: the pass's error word is set, the entry point
reports the failure, the kernel has returned, and the device goes on working."""
import time

import numpy as np
import pytest

import oracle
import sadcs_b200 as sa
from sadcs_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_look_back_gives_up_and_the_device_goes_on():
    limit = 20_000_000  # SM cycles: about 10 ms at 1.965 GHz
    sa.build(np.frombuffer(b"warm up", np.uint8))  # module load and first-use costs out of the timing
    start = time.perf_counter()
    status, word, message = sa.test_lookback_timeout(limit)
    seconds = time.perf_counter() - start
    assert status == sa.GpuStatus.Failed
    assert word == 1 and "gave up" in message
    assert seconds < 2.0  # the wait ended at its limit, far below the production limit of ~2 s
    # the context is intact: a construction right after it is correct
    text = W.random_text(W.SplitMix(8), 50_000, 4)
    suffixes, bwt, primary = sa.build(text)
    expected = oracle.doubling_sa(text)
    assert np.array_equal(suffixes, expected)
    eb, ep = oracle.bwt_from_sa(text, expected)
    assert primary == ep and np.array_equal(bwt, eb)


def test_limit_out_of_range_is_refused():
    status, word, message = sa.test_lookback_timeout(0)
    assert status == sa.GpuStatus.Failed and word == 0 and "out of range" in message
