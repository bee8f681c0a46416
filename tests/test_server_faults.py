"""Error paths of the serving loop (sadcs_gpu_server_*), made on the host: a construction whose
device allocation fails (a fake of the pool's allocation returning out-of-memory), and a request
cancelled while it waits in the queue. Each failure reaches only its own requests; the server goes
on, and every other result still equals the oracle's. No GPU fault is involved."""
import numpy as np
import pytest

import oracle
import sadcs_b200 as sa
from sadcs_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _expected(text):
    s = oracle.doubling_sa(text)
    b, p = oracle.bwt_from_sa(text, s)
    return s, b, p


def _check(result, text):
    s_, b_, p_, _, _ = result
    es, eb, ep = _expected(text)
    assert np.array_equal(s_, es) and np.array_equal(b_, eb) and p_ == ep


def test_failed_allocation_fails_its_request_and_the_server_goes_on():
    with sa.Server(workers=1, small_limit=1 << 20, batch_bytes=16 << 20, batch_texts=64) as server:
        first = W.natural_text(100_000, seed=41)
        second = W.random_text(W.SplitMix(42), 50_000, 20)
        server.fail_allocations(1)
        with pytest.raises(sa.GpuError) as err:
            server.wait(server.submit(first))
        assert err.value.status == sa.GpuStatus.NotEnoughMemory
        assert "allocating from the pool" in str(err.value)
        _check(server.wait(server.submit(second)), second)
        _check(server.wait(server.submit(first)), first)  # the same text again, now allocated


def test_failed_allocation_in_a_mix_reaches_only_its_batch():
    texts = [W.random_text(W.SplitMix(60 + i), 2000 + 97 * i, (4, 20, 256)[i % 3]) for i in range(24)]
    with sa.Server(workers=2, small_limit=1 << 16, batch_bytes=1 << 20, batch_texts=8) as server:
        server.fail_allocations(1)
        tickets = [server.submit(t) for t in texts]
        failed = 0
        for ticket, text in zip(tickets, texts):
            try:
                result = server.wait(ticket)
            except sa.GpuError as e:
                assert e.status == sa.GpuStatus.NotEnoughMemory
                failed += 1
                continue
            _check(result, text)
        assert 1 <= failed <= 8  # the requests of exactly one construction (a batch holds at most 8)


def test_cancel_takes_a_queued_request_only():
    # One worker, busy with 64 MiB of text (tens of milliseconds with its upload from pageable
    # memory); the small requests submitted after it wait in the queue, where one is cancelled.
    big = W.uniform_bytes(64 << 20, seed=7)
    smalls = [W.random_text(W.SplitMix(70 + i), 1000 + 37 * i, 4) for i in range(4)]
    with sa.Server(workers=1, small_limit=1 << 16, batch_bytes=1 << 20, batch_texts=16) as server:
        kb = server.submit(big)
        ks = [server.submit(t) for t in smalls]
        assert server.cancel(ks[1])
        assert not server.cancel(ks[1] + 1000)  # unknown ticket
        with pytest.raises(sa.GpuError) as err:
            server.wait(ks[1])
        assert "cancelled" in str(err.value)
        assert not server.cancel(ks[1])  # waited for: unknown now
        for k, text in zip(ks, smalls):
            if k != ks[1]:
                _check(server.wait(k), text)
        s_, b_, p_, _, _ = server.wait(kb)
        assert not server.cancel(kb)
    alone_sa, alone_bwt, alone_primary = sa.build(big)  # the same text built alone
    assert np.array_equal(s_, alone_sa) and np.array_equal(b_, alone_bwt) and p_ == alone_primary
