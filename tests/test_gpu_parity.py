"""GPU construction vs. the oracle, bit for bit: the cases of the reference's runGpuCases
(src/cli/selftest.cpp:543-606) and testGpuSampleRanks (:474-500), through the C ABI.

The expected SA is the oracle's independent prefix-doubling construction (oracle/dcsa.c), itself
pinned to the reference's own CPU output by tests/test_oracle.py; the expected BWT and sample ranks
are derived from it in the reference's conventions (selftest.cpp:141-159, gpusa.h:65-73).
"""
import numpy as np
import pytest

import oracle
import sadcs_b200 as sa
from sadcs_b200 import workloads as W

pytestmark = pytest.mark.gpu

LARGE = 1 << 22


def _check(text, context=None, name=""):
    text = np.asarray(text, dtype=np.uint8)
    n = len(text)
    expected = oracle.doubling_sa(text)
    got = sa.suffix_array(text, context=context)
    assert got.dtype == np.int32 and len(got) == n
    mismatch = np.nonzero(got.astype(np.uint32) != expected)[0]
    assert mismatch.size == 0, f"{name}: SA differs at {mismatch[:5]} (n={n})"
    eb, ep = oracle.bwt_from_sa(text, expected)
    # The BWT in place of a copy of the text, as `sadcs build --bwt --gpu` does it.
    bwt, primary = sa.bwt(text, context=context)
    assert primary == ep, f"{name}: primary {primary}, expected {ep}"
    assert np.array_equal(bwt, eb), f"{name}: BWT differs at {np.nonzero(bwt != eb)[0][:5]}"
    # Both from one construction.
    s2, b2, p2 = sa.build(text, context=context)
    assert np.array_equal(s2, expected) and np.array_equal(b2, eb) and p2 == ep, f"{name}: build() differs"


def _check_ranks(text, name=""):
    text = np.asarray(text, dtype=np.uint8)
    expected = oracle.sample_ranks_from_sa(oracle.doubling_sa(text), len(text))
    got = sa.rank_sample(text)
    assert np.array_equal(got, expected), f"{name}: sample ranks differ at {np.nonzero(got != expected)[0][:5]}"


WORDS = [b"", b"a", b"banana", b"mississippi", b"abracadabra", b"yabbadabbado"]


@pytest.mark.parametrize("word", WORDS)
def test_words(word):
    _check(np.frombuffer(word, np.uint8), name=repr(word))


def test_runs_and_binary_up_to_80():
    rng = W.SplitMix(3)
    for n in range(0, 81):
        _check(W.run_text(n), name=f"run n={n}")
        _check(W.random_text(rng, n, 2), name=f"sigma=2 n={n}")


def test_sample_ranks_up_to_80():
    rng = W.SplitMix(5)
    for n in range(1, 81):
        _check_ranks(W.run_text(n), name=f"run n={n}")
        _check_ranks(W.random_text(rng, n, 2), name=f"sigma=2 n={n}")


def test_structured():
    rng = W.SplitMix(3)
    _check(W.run_text(1000), name="run 1000")
    _check(W.fibonacci_text(5000), name="fibonacci")
    _check(W.fibonacci_text(5000, 0, 1), name="fibonacci 0/1")
    _check(W.thue_morse_text(4096), name="thue-morse")
    _check(np.zeros(1000, np.uint8), name="zeros")
    run_b = W.run_text(2000)
    run_b[-1] = ord("b")
    _check(run_b, name="run then b")
    b_run = W.run_text(2000)
    b_run[0] = ord("b")
    _check(b_run, name="b then run")
    for period in (1, 2, 3, 5, 7, 31, 32, 33, 63, 64, 65, 1000):
        _check(W.periodic_text(rng, 5000, period), name=f"period {period}")


@pytest.mark.parametrize("sigma", [1, 2, 4, 26, 256])
def test_random_alphabets(sigma):
    rng = W.SplitMix(100 + sigma)
    for i in range(10):
        n = 1 + int(rng.below(20000)[0])
        _check(W.random_text(rng, n, sigma), name=f"sigma={sigma} #{i}")


def test_sample_ranks_structured():
    rng = W.SplitMix(9)
    for period in (1, 2, 3, 7, 31, 32, 33, 64, 65, 1000):
        _check_ranks(W.periodic_text(rng, 5000, period), name=f"period {period}")
    _check_ranks(np.frombuffer(b"banana", np.uint8), name="banana")
    _check_ranks(W.fibonacci_text(5000, 0, 1), name="fibonacci 0/1")
    _check_ranks(W.thue_morse_text(4096), name="thue-morse")
    _check_ranks(W.random_text(rng, 5000, 256), name="sigma=256")


@pytest.mark.parametrize("kind", ["run", "period33", "fibonacci", "thue-morse", "sigma4", "sigma256"])
def test_large(kind):
    rng = W.SplitMix(11)
    text = {
        "run": lambda: W.run_text(LARGE),
        "period33": lambda: W.periodic_text(rng, LARGE, 33),
        "fibonacci": lambda: W.fibonacci_text(LARGE),
        "thue-morse": lambda: W.thue_morse_text(LARGE),
        "sigma4": lambda: W.random_text(rng, LARGE, 4),
        "sigma256": lambda: W.random_text(rng, LARGE, 256),
    }[kind]()
    _check(text, name=f"large {kind}")
    _check_ranks(text, name=f"large {kind}")


def test_carried_words(monkeypatch):
    """Constructions that hand each suffix's first code word from class to class instead of the
    final merge gathering it (one text, codes of at most 2 bits; on their own only from 256 MiB on),
    forced on small texts: the SA, BWT and primary index stay the oracle's. Texts of wider codes take
    the gathering path under the same setting."""
    monkeypatch.setenv("SADCS_CARRY_MIN_BYTES", "0")
    rng = W.SplitMix(21)
    for word in (b"a", b"ab", b"ba", b"banana", b"mississippi", b"acgt" * 9, b"abracadabra"):
        _check(np.frombuffer(word, np.uint8), name=f"carry {word!r}")
    for n in range(0, 81):
        _check(W.run_text(n), name=f"carry run n={n}")
        _check(W.random_text(rng, n, 2), name=f"carry sigma=2 n={n}")
        _check(W.random_text(rng, n, 4), name=f"carry sigma=4 n={n}")
    _check(W.fibonacci_text(5000), name="carry fibonacci")
    _check(W.thue_morse_text(4096), name="carry thue-morse")
    _check(np.zeros(1000, np.uint8), name="carry zeros")
    for i in range(6):
        n = 1 + int(rng.below(40000)[0])
        _check(W.random_text(rng, n, 2 + i % 3), name=f"carry sigma={2 + i % 3} #{i}")
    _check(W.run_text(LARGE), name="carry large run")
    _check(W.fibonacci_text(LARGE), name="carry large fibonacci")
    _check(W.random_text(rng, LARGE, 4), name="carry large sigma=4")
    _check(W.genome_text(LARGE, seed=5), name="carry genome-like 4M")
    with sa.Context(20_000_000) as ctx:
        _check(W.random_text(rng, 20_000_000, 4), context=ctx, name="carry context sigma=4 20M")
        _check(W.random_text(rng, LARGE, 3), context=ctx, name="carry context sigma=3")


def test_context_reuse_and_refusal():
    """selftest.cpp:505-541: one context, largest input first, empties, a refusal, then reuse."""
    rng = W.SplitMix(3)
    capacity = 20_000_000
    with sa.Context(capacity) as ctx:
        assert ctx.capacity == capacity
        _check(W.random_text(rng, capacity, 4), context=ctx, name="context sigma=4 20M")
        _check(W.random_text(rng, LARGE, 256), context=ctx, name="context sigma=256")
        _check(np.frombuffer(b"banana", np.uint8), context=ctx, name="context banana")
        _check(np.zeros(0, np.uint8), context=ctx, name="context empty")
        _check(np.frombuffer(b"a", np.uint8), context=ctx, name="context a")
        _check(W.fibonacci_text(LARGE), context=ctx, name="context fibonacci")
        _check(W.periodic_text(rng, 5000, 33), context=ctx, name="context period 33")
        for i in range(5):
            _check(W.random_text(rng, 1 + int(rng.below(20000)[0]), 2), context=ctx, name=f"context sigma=2 #{i}")
        with pytest.raises(sa.GpuError) as err:
            sa.suffix_array(W.run_text(capacity + 1), context=ctx)
        assert err.value.status == sa.GpuStatus.NotEnoughMemory
        _check(W.random_text(rng, 5000, 26), context=ctx, name="context after refusal")


def test_device_resident_and_gather():
    """build_device on torch-owned HBM buffers, and the SA-to-BWT gather on its output."""
    import torch

    text = W.natural_text(1 << 20, seed=5)
    n = len(text)
    expected = oracle.doubling_sa(text)
    eb, ep = oracle.bwt_from_sa(text, expected)
    d_text = torch.from_numpy(text).cuda()
    d_sa = torch.empty(n, dtype=torch.int32, device="cuda")
    d_bwt = torch.empty(n, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    with sa.Context(n) as ctx:
        primary = sa.build_device(d_text.data_ptr(), n, d_sa.data_ptr(), d_bwt.data_ptr(), context=ctx, stream=stream)
    torch.cuda.synchronize()
    assert primary == ep
    assert np.array_equal(d_sa.cpu().numpy().view(np.uint32), expected)
    assert np.array_equal(d_bwt.cpu().numpy(), eb)
    d_bwt2 = torch.zeros(n, dtype=torch.uint8, device="cuda")
    p2 = sa.bwt_from_sa_device(d_text.data_ptr(), n, d_sa.data_ptr(), d_bwt2.data_ptr(), stream=stream)
    torch.cuda.synchronize()
    assert p2 == ep and np.array_equal(d_bwt2.cpu().numpy(), eb)


def _expected(text):
    sa_ = oracle.doubling_sa(text)
    b, p = oracle.bwt_from_sa(text, sa_)
    return sa_, b, p


def test_batch_matches_single_texts():
    """One construction of many uneven texts: every text's SA and BWT bit-exact with its own."""
    rng = W.SplitMix(41)
    texts = [np.frombuffer(b"banana", np.uint8), np.zeros(0, np.uint8), np.frombuffer(b"a", np.uint8),
             W.run_text(100), W.fibonacci_text(3000), W.periodic_text(rng, 5000, 33), np.zeros(700, np.uint8)]
    for i in range(40):
        n = 1 + int(rng.below(6000)[0])
        texts.append(W.random_text(rng, n, [1, 2, 4, 26, 256][i % 5]))
    texts += W.batch_texts(24, lo=1 << 10, hi=1 << 17, seed=8)
    sas, bwts, primaries = sa.build_batch(texts)
    for j, t in enumerate(texts):
        es, eb, ep = _expected(t)
        assert np.array_equal(sas[j], es), f"text {j} (n={len(t)}): SA differs"
        assert np.array_equal(bwts[j], eb) and primaries[j] == ep, f"text {j} (n={len(t)}): BWT differs"


def test_batch_context_reuse_and_device_path():
    import torch

    texts = W.batch_texts(64, lo=1 << 10, hi=1 << 16, seed=9)
    lengths = [len(t) for t in texts]
    total = sum(lengths)
    with sa.Context(total, max_texts=64) as ctx:
        for _ in range(2):
            sas, bwts, primaries = sa.build_batch(texts, context=ctx)
            for j, t in enumerate(texts):
                es, eb, ep = _expected(t)
                assert np.array_equal(sas[j], es) and np.array_equal(bwts[j], eb) and primaries[j] == ep
        packed = torch.from_numpy(np.concatenate(texts)).cuda()
        d_sa = torch.empty(total, dtype=torch.int32, device="cuda")
        d_bwt = torch.empty(total, dtype=torch.uint8, device="cuda")
        prim = sa.build_batch_device(packed.data_ptr(), lengths, d_sa.data_ptr(), d_bwt.data_ptr(), context=ctx,
                                     stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        all_sa = d_sa.cpu().numpy().view(np.uint32)
        all_bwt = d_bwt.cpu().numpy()
        off = np.concatenate([[0], np.cumsum(lengths)])
        for j, t in enumerate(texts):
            es, eb, ep = _expected(t)
            assert np.array_equal(all_sa[off[j]:off[j + 1]], es) and np.array_equal(all_bwt[off[j]:off[j + 1]], eb)
            assert prim[j] == ep
        with pytest.raises(sa.GpuError) as err:
            sa.build_batch(texts + [W.run_text(10)], context=ctx)
        assert err.value.status == sa.GpuStatus.NotEnoughMemory


def test_server_results_equal_alone_and_in_the_mix():
    """Continuous batching: requests submitted while others run; each result equals its own build."""
    import threading
    import time

    rng = np.random.default_rng(12)
    texts = W.batch_texts(60, lo=1 << 10, hi=1 << 18, seed=12) + [W.natural_text(3 << 20, seed=13),
                                                                 W.run_text(5000), np.zeros(0, np.uint8)]
    order = rng.permutation(len(texts))
    with sa.Server(workers=3, small_limit=1 << 20, batch_bytes=16 << 20, batch_texts=64) as server:
        tickets = {}

        def producer():
            for k in order:
                tickets[int(k)] = server.submit(texts[int(k)])
                time.sleep(0.001)

        thread = threading.Thread(target=producer)
        thread.start()
        thread.join()
        batched = 0
        for k, ticket in tickets.items():
            s_, b_, p_, latency, size = server.wait(ticket)
            es, eb, ep = _expected(texts[k])
            assert np.array_equal(s_, es) and np.array_equal(b_, eb) and p_ == ep, f"request {k} differs"
            assert latency[2] >= latency[1] >= 0
            batched += size > 1
        assert batched > 0  # some requests shared a construction
        constructions, launches = server.counters()
        assert 0 < constructions < len(texts) and launches > 0


@pytest.mark.parametrize("mode", ["overlapped", "mapped", "after"])
@pytest.mark.parametrize("n", [1, 2, 100, 70000, 3 << 20])
def test_page_locked_outputs(n, mode, monkeypatch):
    """Page-locked output buffers: copied down piece by piece while the last merge level runs (the
    default: each piece up to the window base of the next piece's first tile), written by the merge
    itself through their device mapping, or copied after the construction. The results equal those
    of the pageable path, for natural-language-like text and for DNA-like text with carried words
    (pieces of SA only, BWT only, and both)."""
    rng = W.SplitMix(n)
    texts = [W.natural_text(n, seed=31) if n > 100 else W.random_text(rng, n, 3), W.random_text(rng, n, 4)]
    monkeypatch.setenv("SADCS_CARRY_MIN_BYTES", "0")
    raw_sa = sa.allocate_pinned(4 * n)
    raw_bwt = sa.allocate_pinned(n)
    try:
        for text in texts:
            monkeypatch.setenv("SADCS_HOST_OUTPUTS", "after")
            ref_sa, ref_bwt, ref_primary = sa.build(text)
            monkeypatch.setenv("SADCS_HOST_OUTPUTS", mode)
            out_sa = raw_sa.view(np.uint32)
            for want_sa, want_bwt in ((True, True), (True, False), (False, True)):
                out_sa[:] = 0xFFFFFFFF
                raw_bwt[:] = 0
                got_sa, got_bwt, primary = sa.build(text, want_sa=want_sa, want_bwt=want_bwt,
                                                    out_sa=out_sa if want_sa else None,
                                                    out_bwt=raw_bwt if want_bwt else None)
                if want_sa:
                    assert np.array_equal(got_sa, ref_sa), f"{mode}: SA differs (n={n})"
                if want_bwt:
                    assert np.array_equal(got_bwt, ref_bwt) and primary == ref_primary, f"{mode}: BWT differs (n={n})"
    finally:
        sa.free_pinned(raw_sa)
        sa.free_pinned(raw_bwt)


@pytest.mark.parametrize("mode", ["overlapped", "mapped", "after"])
def test_page_locked_outputs_of_a_batch(mode, monkeypatch):
    """A batch of uneven texts into page-locked buffers (all texts one after another): the pieces
    copied down while the last merge level runs follow the global output order across texts; every
    text's SA, BWT and primary equal its own construction's."""
    monkeypatch.setenv("SADCS_HOST_OUTPUTS", mode)
    texts = W.batch_texts(60, lo=1 << 8, hi=1 << 18, seed=22) + [W.natural_text(1 << 20, seed=23)]
    total = sum(len(t) for t in texts)
    raw_sa = sa.allocate_pinned(4 * total)
    raw_bwt = sa.allocate_pinned(total)
    try:
        out_sa = raw_sa.view(np.uint32)
        out_sa[:] = 0xFFFFFFFF
        raw_bwt[:] = 0
        sas, bwts, primaries = sa.build_batch(texts, out_sa=out_sa, out_bwt=raw_bwt)
        for k, t in enumerate(texts):
            es, eb, ep = _expected(t)
            assert np.array_equal(sas[k], es) and np.array_equal(bwts[k], eb) and primaries[k] == ep, \
                f"{mode}: text {k} differs"
    finally:
        sa.free_pinned(raw_sa)
        sa.free_pinned(raw_bwt)


def test_server_carried_words(monkeypatch):
    """Requests built alone by the server (one text per construction) with carried words forced on
    (normally from 256 MiB on): the server plans the room for them in a request's footprint and its
    construction uses it; results equal the oracle's, pageable and page-locked outputs alike."""
    monkeypatch.setenv("SADCS_CARRY_MIN_BYTES", "0")
    rng = W.SplitMix(24)
    texts = [W.random_text(rng, n, 4) for n in (1000, 70000, 1 << 20)] + [W.genome_text(1 << 21, seed=7),
                                                                             W.random_text(rng, 5000, 2)]
    raw = sa.allocate_pinned(sum(5 * len(t) + 64 for t in texts))
    try:
        with sa.Server(workers=2, small_limit=1 << 20, batch_bytes=64 << 20, batch_texts=1) as server:
            tickets, at = [], 0
            for k, t in enumerate(texts):
                n = len(t)
                if k % 2:
                    out_sa = raw[at:at + 4 * n].view(np.uint32)
                    at += (4 * n + 15) // 16 * 16
                    out_bwt = raw[at:at + n]
                    at += (n + 15) // 16 * 16
                    tickets.append(server.submit(t, sa=out_sa, bwt=out_bwt))
                else:
                    tickets.append(server.submit(t))
            for k, ticket in enumerate(tickets):
                s_, b_, p_, _, size = server.wait(ticket)
                es, eb, ep = _expected(texts[k])
                assert size == 1
                assert np.array_equal(s_, es) and np.array_equal(b_, eb) and p_ == ep, f"request {k} differs"
    finally:
        sa.free_pinned(raw)


def test_server_page_locked_outputs_in_batches():
    """Requests whose outputs are page-locked: the batched merge writes each request's SA and BWT
    into that request's own buffers; every result equals its text built alone."""
    texts = W.batch_texts(40, lo=1 << 10, hi=1 << 17, seed=14) + [W.natural_text(1 << 20, seed=15)]
    lengths = [len(t) for t in texts]
    raw = sa.allocate_pinned(sum(5 * n + 64 for n in lengths))
    try:
        views, at = [], 0
        for n in lengths:
            out_sa = raw[at:at + 4 * n].view(np.uint32)
            at += (4 * n + 15) // 16 * 16
            out_bwt = raw[at:at + n]
            at += (n + 15) // 16 * 16
            out_sa[:] = 0xFFFFFFFF
            views.append((out_sa, out_bwt))
        with sa.Server(workers=2, small_limit=1 << 20, batch_bytes=64 << 20, batch_texts=64) as server:
            tickets = [server.submit(t, sa=v[0], bwt=v[1]) for t, v in zip(texts, views)]
            batched = 0
            for k, ticket in enumerate(tickets):
                s_, b_, p_, _, size = server.wait(ticket)
                es, eb, ep = _expected(texts[k])
                assert np.array_equal(s_, es) and np.array_equal(b_, eb) and p_ == ep, f"request {k} differs"
                batched += size > 1
            assert batched > 0
    finally:
        sa.free_pinned(raw)
