"""Seeded synthetic texts: the adversarial families of the reference's selftest and the benchmark shapes.

The reference's benchmark corpora (Silesia, enwik8/9, Pizza&Chili) are not available offline; the
generators below produce seeded stand-ins with the shapes, sizes and value distributions of the
workloads this library is measured on:

* ``uniform_bytes``      8 MiB i.i.d. uniform bytes (the reference's CPU-runnable case)
* ``natural_text``       natural-language-like text: a 50k-word lowercase vocabulary, word lengths
                         uniform in 2-12, words drawn Zipf(s=1.1), single spaces, ".\\n" every 10-30
                         words (uniform), 2% of words capitalised
* ``genome_text``        {A,C,G,T} text: a prefix of 2/3 i.i.d. with GC fraction 0.41, then copies of
                         randomly chosen 1 MiB segments of that prefix with 1% point substitutions
                         and 0.1% indels of 1-10 characters
* ``batch_texts``        many texts with log-uniform lengths over three alphabets (DNA, protein-like,
                         uniform bytes)

The selftest families (src/cli/selftest.cpp:31-108 of the reference) are restated for the
adversarial parity cases: splitmix64 random text over small alphabets, periodic text, Fibonacci
words, Thue-Morse words and runs.
"""
from __future__ import annotations

import numpy as np

_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, count: int, offset: int = 0) -> np.ndarray:
    """The first ``count`` outputs (after ``offset``) of splitmix64 seeded with ``seed``.

    Output i is mix(seed + (i + 1) * gamma): the generator's state advances by a constant, so the
    stream vectorises.
    """
    with np.errstate(over="ignore"):
        idx = np.arange(offset + 1, offset + count + 1, dtype=np.uint64)
        z = np.uint64(seed) + idx * _GAMMA
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


class SplitMix:
    """Sequential splitmix64 (selftest.cpp:31-44), for cases that consume the stream in calls."""

    def __init__(self, seed: int):
        self.seed = int(seed)
        self.used = 0

    def take(self, count: int) -> np.ndarray:
        out = splitmix64(self.seed, count, self.used)
        self.used += count
        return out

    def below(self, bound: int, count: int = 1) -> np.ndarray:
        return (self.take(count) % np.uint64(bound)).astype(np.uint32)


def random_text(rng: SplitMix, n: int, sigma: int) -> np.ndarray:
    """sigma == 256: uniform bytes; otherwise 'a' + uniform below sigma (selftest.cpp:63-71)."""
    v = rng.below(sigma, n)
    return (v if sigma == 256 else v + ord("a")).astype(np.uint8)


def periodic_text(rng: SplitMix, n: int, period: int) -> np.ndarray:
    pattern = random_text(rng, period, 4)
    return np.resize(pattern, n).astype(np.uint8)


def fibonacci_text(n: int, a: int = ord("a"), b: int = ord("b")) -> np.ndarray:
    shorter = np.array([a], np.uint8)
    longer = np.array([a, b], np.uint8)
    while len(longer) < n:
        shorter, longer = longer, np.concatenate([longer, shorter])
    return longer[:n].copy()


def thue_morse_text(n: int) -> np.ndarray:
    i = np.arange(n, dtype=np.uint64)
    parity = np.zeros(n, np.uint8)
    for bit in range(64):
        parity ^= ((i >> np.uint64(bit)) & np.uint64(1)).astype(np.uint8)
        if n <= (1 << (bit + 1)):
            break
    return (parity + ord("a")).astype(np.uint8)


def run_text(n: int, c: int = ord("a")) -> np.ndarray:
    return np.full(n, c, np.uint8)


# ---- benchmark shapes ------------------------------------------------------------------------

def uniform_bytes(n: int = 8 << 20, seed: int = 1) -> np.ndarray:
    return np.random.default_rng(seed).integers(0, 256, n, dtype=np.uint8)


def natural_text(n: int = 256 << 20, seed: int = 2, vocabulary: int = 50_000, zipf_s: float = 1.1,
                 capital_fraction: float = 0.02) -> np.ndarray:
    rng = np.random.default_rng(seed)
    lengths = rng.integers(2, 13, vocabulary)
    letters = rng.integers(ord("a"), ord("z") + 1, int(lengths.sum()), dtype=np.uint8)
    word_start = np.concatenate([[0], np.cumsum(lengths)[:-1]])
    weights = 1.0 / np.arange(1, vocabulary + 1, dtype=np.float64) ** zipf_s
    cdf = np.cumsum(weights / weights.sum())
    mean_len = float((weights / weights.sum() * lengths).sum()) + 1.1
    out = np.empty(n, np.uint8)
    filled = 0
    until_stop = int(rng.integers(10, 31))
    while filled < n:
        count = int((n - filled) / mean_len * 1.05) + 64
        words = np.minimum(np.searchsorted(cdf, rng.random(count)), vocabulary - 1)
        wl = lengths[words]
        # Sentence ends: ".\n" after every U[10,30] words, a space otherwise.
        ends = until_stop - 1 + np.concatenate([[0], np.cumsum(rng.integers(10, 31, count // 10 + 2))])
        inside = ends[ends < count]
        until_stop = int(ends[len(inside)]) - count + 1
        stop = np.zeros(count, bool)
        stop[inside] = True
        sep_len = np.where(stop, 2, 1)
        total = wl + sep_len
        offs = np.concatenate([[0], np.cumsum(total)[:-1]])
        chunk = np.empty(int(total.sum()), np.uint8)
        # Scatter every word's letters.
        idx_in_word = np.arange(int(wl.sum())) - np.repeat(np.cumsum(wl) - wl, wl)
        src = np.repeat(word_start[words], wl) + idx_in_word
        dst = np.repeat(offs, wl) + idx_in_word
        chunk[dst] = letters[src]
        cap = rng.random(count) < capital_fraction
        chunk[offs[cap]] -= 32
        sep_at = offs + wl
        chunk[sep_at] = np.where(stop, ord("."), ord(" ")).astype(np.uint8)
        chunk[(sep_at + 1)[stop]] = ord("\n")
        take = min(n - filled, len(chunk))
        out[filled:filled + take] = chunk[:take]
        filled += take
    return out


_DNA = np.frombuffer(b"ACGT", np.uint8)


def _iid_dna(rng: np.random.Generator, n: int, gc: float = 0.41, out: np.ndarray | None = None) -> np.ndarray:
    out = np.empty(n, np.uint8) if out is None else out
    cdf = np.cumsum([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    chunk = 1 << 20  # small temporaries are reused by the allocator instead of faulted in afresh
    c = cdf.astype(np.float32)
    for s in range(0, n, chunk):
        u = rng.random(min(chunk, n - s), dtype=np.float32)
        # letter index = how many of the first three cdf entries are <= u (u < 1 = the last entry)
        index = (u >= c[0]).view(np.uint8) + (u >= c[1]).view(np.uint8) + (u >= c[2]).view(np.uint8)
        out[s:s + len(u)] = _DNA[index]
    return out


def genome_text(n: int = 3 << 30, seed: int = 3, segment: int = 1 << 20, substitution: float = 0.01,
                indel: float = 0.001, prefix: int | None = None) -> np.ndarray:
    """2/3 i.i.d. DNA (GC 0.41), then mutated copies of random ``segment``-long pieces of it.

    ``prefix`` <= 2n/3: only the first ``prefix`` bytes of that text (the i.i.d. part is one
    sequential stream, so they come out the same without generating the rest)."""
    rng = np.random.default_rng(seed)
    base_len = (n * 2) // 3
    if prefix is not None and prefix <= base_len:
        return _iid_dna(rng, prefix)
    out = np.empty(n, np.uint8)
    _iid_dna(rng, base_len, out=out[:base_len])
    filled = base_len
    while filled < n:
        start = int(rng.integers(0, max(1, base_len - segment)))
        piece = out[start:start + segment].copy()
        subs = np.nonzero(rng.random(len(piece), dtype=np.float32) < substitution)[0]
        piece[subs] = _DNA[(np.searchsorted(_DNA, piece[subs]) + rng.integers(1, 4, len(subs))) % 4]
        events = np.nonzero(rng.random(len(piece), dtype=np.float32) < indel)[0]
        if len(events):
            parts = []
            prev = 0
            for e in events:
                e = int(e)
                if e < prev:
                    continue
                length = int(rng.integers(1, 11))
                parts.append(piece[prev:e])
                if rng.random() < 0.5:  # insertion
                    parts.append(_DNA[rng.integers(0, 4, length)])
                    prev = e
                else:  # deletion
                    prev = e + length
            parts.append(piece[prev:])
            piece = np.concatenate(parts)
        take = min(n - filled, len(piece))
        out[filled:filled + take] = piece[:take]
        filled += take
    return out


# Background amino-acid frequencies (percent), alphabetical by one-letter code.
_AMINO = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWY", np.uint8)
_AMINO_FREQ = np.array([8.25, 1.37, 5.45, 6.75, 3.86, 7.07, 2.27, 5.96, 5.84, 9.66,
                        2.42, 4.06, 4.70, 3.93, 5.53, 6.56, 5.34, 6.87, 1.08, 2.92])


def protein_text(rng: np.random.Generator, n: int) -> np.ndarray:
    p = _AMINO_FREQ / _AMINO_FREQ.sum()
    return _AMINO[np.searchsorted(np.cumsum(p), rng.random(n), side="right").clip(0, 19)]


def batch_lengths(count: int = 4096, lo: int = 1 << 10, hi: int = 4 << 20, seed: int = 4) -> np.ndarray:
    """Lengths of a batch: log-uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(np.int64)


def batch_text(index: int, n: int, seed: int = 4) -> np.ndarray:
    """Text ``index`` of a batch (its own generator, so any subset can be made alone): DNA,
    protein-like and uniform bytes by index mod 3."""
    rng = np.random.default_rng([seed, index])
    kind = index % 3
    if kind == 0:
        return _DNA[rng.integers(0, 4, int(n))]
    if kind == 1:
        return protein_text(rng, int(n))
    return rng.integers(0, 256, int(n), dtype=np.uint8)


def batch_texts(count: int = 4096, lo: int = 1 << 10, hi: int = 4 << 20, seed: int = 4, indices=None):
    """``count`` texts, lengths log-uniform in [lo, hi]; thirds over DNA, protein-like, uniform bytes.
    ``indices`` picks a subset (in the given order)."""
    lengths = batch_lengths(count, lo, hi, seed)
    picked = range(count) if indices is None else indices
    return [batch_text(i, int(lengths[i]), seed) for i in picked]


def partition_by_footprint(lengths, parts: int) -> list[list[int]]:
    """Greedy longest-first bin packing of texts onto ``parts`` devices by construction footprint
    (proportional to length): each text, longest first, goes to the least-loaded part. Every index
    lands in exactly one part; each part keeps its indices in ascending order."""
    order = sorted(range(len(lengths)), key=lambda i: (-int(lengths[i]), i))
    loads = [0] * parts
    out: list[list[int]] = [[] for _ in range(parts)]
    for i in order:
        k = min(range(parts), key=lambda q: (loads[q], q))
        out[k].append(i)
        loads[k] += int(lengths[i])
    return [sorted(x) for x in out]
