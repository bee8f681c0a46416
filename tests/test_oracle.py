"""The oracle (oracle/dcsa.c) pinned to the reference's own outputs (tests/golden/, made by
tests/golden/make_golden.py from the reference's CPU build), and the checker's planted-error suite
of the reference's selftest (src/cli/selftest.cpp:309-385). CPU only."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from sadcs_b200 import workloads as W
from tests.golden.make_golden import small_inputs

GOLDEN = Path(__file__).resolve().parent / "golden"


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _small_cases():
    cases = json.loads((GOLDEN / "small.json").read_text())["cases"]
    inputs = dict(small_inputs())
    return [(c, inputs[c["name"]]) for c in cases]


SMALL = _small_cases()


@pytest.mark.parametrize("case,text", SMALL, ids=[c["name"] for c, _ in SMALL])
def test_oracle_matches_reference_small(case, text):
    assert digest(text) == case["text_sha256"], "generator drifted from the golden inputs"
    if "text" in case:
        assert text.tobytes().hex() == case["text"]
    for construct in (oracle.naive_sa, oracle.doubling_sa, oracle.dc_sa):
        sa = construct(text)
        assert digest(sa.astype("<i4")) == case["sa_sha256"], construct.__name__
        if "sa" in case:
            assert sa.tolist() == case["sa"]
    bwt, primary = oracle.bwt_from_sa(text, oracle.doubling_sa(text))
    assert primary == case["primary"] and digest(bwt) == case["bwt_sha256"]
    assert oracle.check_sa(text, oracle.doubling_sa(text))[0]
    assert oracle.check_bwt(text, bwt, primary)[0]


LARGE = json.loads((GOLDEN / "large.json").read_text())["cases"]


@pytest.mark.parametrize("case", LARGE, ids=[c["name"] for c in LARGE])
def test_oracle_matches_reference_large(case):
    text = eval(case["generator"], {"W": W})
    assert len(text) == case["n"] and digest(text) == case["text_sha256"], "generator drifted"
    sa = oracle.doubling_sa(text)
    assert digest(sa.astype("<i4")) == case["sa_sha256"]
    bwt, primary = oracle.bwt_from_sa(text, sa)
    assert primary == case["primary"] and digest(bwt) == case["bwt_sha256"]


@pytest.mark.parametrize("name", ["natural text 4 MiB seed 2", "genome text 6 MiB seed 3"])
def test_dc_restatement_large(name):
    """The DC32 restatement (ranking, classes, merge) on inputs with long repeats."""
    case = next(c for c in LARGE if c["name"] == name)
    text = eval(case["generator"], {"W": W})
    assert digest(oracle.dc_sa(text).astype("<i4")) == case["sa_sha256"]


def test_dc_intermediates():
    """Sample ranks and class lists of the restatement agree with those a suffix array implies."""
    rng = W.SplitMix(17)
    for text in (W.fibonacci_text(3000), W.periodic_text(rng, 4000, 33), W.random_text(rng, 5000, 4),
                 W.natural_text(20000, seed=9), np.frombuffer(b"mississippi", np.uint8)):
        sa = oracle.doubling_sa(text)
        ranks = oracle.dc_sample_ranks(text)
        assert np.array_equal(ranks, oracle.sample_ranks_from_sa(sa, len(text)))
        lists, start = oracle.dc_class_lists(text, ranks)
        lists2, start2 = oracle.class_lists_from_sa(sa, len(text))
        assert np.array_equal(start, start2) and np.array_equal(lists, lists2)


def _mutations():
    return [
        ("swapped neighbours", lambda sa: sa.__setitem__(slice(1000, 1002), sa[1000:1002][::-1].copy())),
        ("swapped far apart", lambda sa: sa.__setitem__([10, 2900], sa[[2900, 10]])),
        ("duplicate entry", lambda sa: sa.__setitem__(500, sa[1500])),
        ("out of range", lambda sa: sa.__setitem__(42, len(sa))),
    ]


def test_checker_catches_planted_errors():
    rng = W.SplitMix(7)
    text = W.random_text(rng, 3000, 3)
    good = oracle.naive_sa(text)
    assert oracle.check_sa(text, good)[0]
    for name, mutate in _mutations():
        bad = good.copy()
        mutate(bad)
        assert not oracle.check_sa(text, bad)[0], name
    bwt, primary = oracle.bwt_from_sa(text, good)
    assert oracle.check_bwt(text, bwt, primary)[0]
    swapped = bwt.copy()
    i = 1000 + int(np.nonzero(swapped[1000:-1] != swapped[1001:])[0][0])
    swapped[i], swapped[i + 1] = swapped[i + 1], swapped[i]
    changed = bwt.copy()
    changed[1234] ^= 1
    for name, b, p in (("swapped neighbours", swapped, primary), ("changed character", changed, primary),
                       ("primary off by one", bwt, primary + 1 if primary < 3000 else primary - 1),
                       ("primary 0", bwt, 0)):
        assert not oracle.check_bwt(text, b, p)[0], name


@pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU build not present")
def test_oracle_vs_reference_random():
    rng = W.SplitMix(99)
    for sigma in (1, 2, 4, 26, 256):
        for _ in range(4):
            text = W.random_text(rng, 1 + int(rng.below(20000)[0]), sigma)
            assert np.array_equal(oracle.dc_sa(text), oracle.ref_sa(text).astype(np.uint32))


def _naive_lcp(text: np.ndarray, sa: np.ndarray) -> np.ndarray:
    out = np.zeros(len(sa), np.uint32)
    for r in range(1, len(sa)):
        a, b = text[int(sa[r - 1]):], text[int(sa[r]):]
        m = min(len(a), len(b))
        differ = np.flatnonzero(a[:m] != b[:m])
        out[r] = differ[0] if len(differ) else m
    return out


def test_lcp_oracle_matches_the_definition():
    """oracle.lcp (Kasai over the Phi array; no reference counterpart) against direct comparison of
    every pair of neighbouring suffixes, on the golden inputs and on run, Fibonacci and natural text."""
    texts = [text for _, text in SMALL]
    texts += [W.run_text(3000), W.fibonacci_text(4000), W.natural_text(6000, seed=4),
              np.frombuffer(b"mississippi", np.uint8), np.frombuffer(b"a", np.uint8)]
    for text in texts:
        text = np.ascontiguousarray(text, dtype=np.uint8)
        if len(text) == 0 or len(text) > 20000:
            continue
        sa = oracle.naive_sa(text)
        assert np.array_equal(oracle.lcp(text, sa), _naive_lcp(text, sa))
    assert len(oracle.lcp(np.zeros(0, np.uint8), np.zeros(0, np.uint32))) == 0
