"""The seeded synthetic workloads stand in for corpora that are not available offline, so their shapes
are part of what the benchmark numbers mean: these tests pin each generator to its stated
distribution (sadcs_b200/workloads.py). CPU only, small sizes."""
import numpy as np

from sadcs_b200 import workloads as W


def test_generators_are_deterministic():
    assert np.array_equal(W.natural_text(1 << 16, seed=2), W.natural_text(1 << 16, seed=2))
    assert not np.array_equal(W.natural_text(1 << 16, seed=2), W.natural_text(1 << 16, seed=3))
    assert np.array_equal(W.genome_text(1 << 16, seed=3, segment=1 << 12), W.genome_text(1 << 16, seed=3, segment=1 << 12))
    assert np.array_equal(W.uniform_bytes(1 << 16, seed=1), W.uniform_bytes(1 << 16, seed=1))
    assert np.array_equal(W.batch_text(7, 5000), W.batch_text(7, 5000))


def test_natural_text_shape():
    """Lowercase words of 2-12 letters, single spaces, '.\\n' after every 10-30 words, about 2% of
    words capitalised, word frequencies Zipf(1.1)."""
    text = W.natural_text(4 << 20, seed=2)
    allowed = set(range(ord("a"), ord("z") + 1)) | set(range(ord("A"), ord("Z") + 1)) | {ord(" "), ord("."), ord("\n")}
    assert set(np.unique(text).tolist()) <= allowed
    s = text.tobytes().decode("ascii")
    sentences = s.split(".\n")[1:-1]  # whole sentences only
    counts = np.array([len(x.split(" ")) for x in sentences])
    assert counts.min() >= 10 and counts.max() <= 30
    assert abs(counts.mean() - 20) < 0.5
    words = " ".join(sentences).split(" ")
    lengths = np.array([len(w) for w in words])
    assert lengths.min() >= 2 and lengths.max() <= 12
    capital = np.mean([w[0].isupper() for w in words])
    assert 0.015 < capital < 0.025
    lower = [w.lower() for w in words]
    _, freq = np.unique(lower, return_counts=True)
    top = np.sort(freq)[::-1]
    # Zipf(1.1): the most frequent word about 2^1.1 = 2.14 times as frequent as the second
    # (capitalised copies are folded in; two words of the random vocabulary may coincide)
    assert 1.7 < top[0] / top[1] < 2.6


def test_genome_text_shape():
    """{A,C,G,T}; the first two thirds i.i.d. with GC 0.41; the last third made of mutated copies of
    segments of the first part (most of its 32-mers occur there, unlike a random text's)."""
    n = 3 << 20
    text = W.genome_text(n, seed=3, segment=1 << 16)
    assert set(np.unique(text).tolist()) <= set(b"ACGT")
    base = text[: 2 * n // 3]
    gc = np.isin(base, np.frombuffer(b"GC", np.uint8)).mean()
    assert abs(gc - 0.41) < 0.005
    code = np.searchsorted(np.frombuffer(b"ACGT", np.uint8), text).astype(np.uint64)

    def kmers(a, k=32):
        out = np.zeros(len(a) - k + 1, np.uint64)
        for i in range(k):
            out = (out << np.uint64(2)) | a[i:len(a) - k + 1 + i]
        return out

    known = np.unique(kmers(code[: 2 * n // 3]))
    rng = np.random.default_rng(0)
    tail = kmers(code[2 * n // 3:])
    sample = tail[rng.integers(0, len(tail), 2000)]
    found = np.isin(sample, known).mean()
    assert found > 0.6  # 0.99^32 intact without indels; an i.i.d. text would give about 0
    fresh = kmers(rng.integers(0, 4, 5000).astype(np.uint64))  # a random text's 32-mers, for contrast
    assert np.isin(fresh, known).mean() < 0.01


def test_genome_prefix_is_the_texts_start():
    """The prefix path (used to sample the 3 GiB text for the CPU baseline without generating all
    of it) gives the same bytes as the whole text's start, across generator chunk boundaries."""
    n = 6 << 20
    text = W.genome_text(n, seed=3, segment=1 << 16)
    for k in (1, 12345, 1 << 20, (1 << 20) + 7, 2 * n // 3):
        assert np.array_equal(W.genome_text(n, seed=3, segment=1 << 16, prefix=k), text[:k])


def test_batch_shapes():
    """4096 lengths log-uniform in [1 KiB, 4 MiB] (mean about 0.48 MiB, about 1.9 GiB in all); texts by
    index mod 3 over DNA, 20 amino acids and uniform bytes."""
    lengths = W.batch_lengths()
    assert len(lengths) == 4096
    assert lengths.min() >= 1 << 10 and lengths.max() <= 4 << 20
    logs = np.log(lengths)
    assert abs(logs.mean() - (np.log(1 << 10) + np.log(4 << 20)) / 2) < 0.1
    assert 1.7 * (1 << 30) < lengths.sum() < 2.2 * (1 << 30)
    assert set(np.unique(W.batch_text(0, 20000)).tolist()) <= set(b"ACGT")
    assert set(np.unique(W.batch_text(1, 20000)).tolist()) <= set(b"ACDEFGHIKLMNPQRSTVWY")
    assert len(np.unique(W.batch_text(2, 200000))) == 256
    picked = W.batch_texts(count=12, lo=100, hi=200, indices=[5, 2])
    assert np.array_equal(picked[0], W.batch_text(5, len(picked[0])))


def test_uniform_bytes_shape():
    counts = np.bincount(W.uniform_bytes(1 << 20, seed=1), minlength=256)
    expected = (1 << 20) / 256
    chi2 = ((counts - expected) ** 2 / expected).sum()
    assert chi2 < 350  # 255 degrees of freedom
