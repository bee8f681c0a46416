"""Generates tests/golden/*.json from the reference's own CPU build (oracle/_ref/libsadcs_ref.so).

Run in a container where the reference sources exist (``make -C oracle ref`` first):

    python tests/golden/make_golden.py

Every input is regenerated from a seeded generator in sadcs_b200.workloads (small_inputs() below,
which the tests import; inputs of up to 300 bytes are also stored verbatim), and the reference's buildSuffixArray / buildBwt (cover 128, its CPU default)
produce the expected outputs: full arrays for inputs of up to 300 bytes, SHA-256 digests of the little-endian
int32 SA and of the BWT bytes for every input. The reference's checker accepts each output.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

import oracle  # noqa: E402
from sadcs_b200 import workloads as W  # noqa: E402


def small_inputs():
    rng = W.SplitMix(21)
    cases = [("word " + w.decode(), np.frombuffer(w, np.uint8).copy())
             for w in (b"", b"a", b"ab", b"ba", b"aa", b"aab", b"banana", b"mississippi", b"abracadabra",
                       b"yabbadabbado")]
    for n in (1, 2, 7, 8, 9, 15, 16, 17, 31, 32, 33, 63, 64, 65, 127, 128, 129, 255, 256, 257, 270):
        cases.append((f"run n={n}", W.run_text(n)))
    cases.append(("zeros 1000", np.zeros(1000, np.uint8)))
    rb = W.run_text(2000)
    rb[-1] = ord("b")
    cases.append(("run then b", rb))
    br = W.run_text(2000)
    br[0] = ord("b")
    cases.append(("b then run", br))
    for period in (1, 2, 3, 5, 7, 31, 32, 33, 63, 64, 65, 127, 128, 129, 255, 256, 257, 1000):
        cases.append((f"period {period}", W.periodic_text(rng, 5000, period)))
    cases.append(("fibonacci", W.fibonacci_text(5000)))
    cases.append(("fibonacci 0/1", W.fibonacci_text(5000, 0, 1)))
    cases.append(("thue-morse", W.thue_morse_text(4096)))
    for sigma in (1, 2, 3, 4, 26, 256):
        for i in range(4):
            n = 1 + int(rng.below(4000)[0])
            cases.append((f"random sigma={sigma} #{i}", W.random_text(rng, n, sigma)))
    return cases


LARGE = [
    # (name, generator expression evaluated with W in scope)
    ("uniform bytes 8 MiB seed 1", "W.uniform_bytes(8 << 20, seed=1)"),
    ("natural text 4 MiB seed 2", "W.natural_text(4 << 20, seed=2)"),
    ("genome text 6 MiB seed 3", "W.genome_text(6 << 20, seed=3, segment=1 << 16)"),
    ("large run 4 MiB", "W.run_text(1 << 22)"),
    ("large fibonacci 4 MiB", "W.fibonacci_text(1 << 22)"),
    ("large thue-morse 4 MiB", "W.thue_morse_text(1 << 22)"),
]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    if not oracle.ref_available():
        sys.exit("oracle/_ref/libsadcs_ref.so is missing: make -C oracle ref")
    small = []
    for name, text in small_inputs():
        sa = oracle.ref_sa(text)
        bwt, primary = oracle.ref_bwt(text)
        assert oracle.ref_check_sa(text, sa)[0] and oracle.ref_check_bwt(text, bwt, primary)[0], name
        case = {"name": name, "n": int(len(text)), "text_sha256": digest(text),
                "sa_sha256": digest(sa.astype("<i4")), "bwt_sha256": digest(bwt), "primary": primary}
        if len(text) <= 300:
            case.update({"text": text.tobytes().hex(), "sa": sa.tolist(), "bwt": bwt.tobytes().hex()})
        small.append(case)
    (HERE / "small.json").write_text(json.dumps({"source": "reference CPU build, cover 128", "cases": small},
                                                indent=0))
    large = []
    for name, expr in LARGE:
        text = eval(expr, {"W": W})
        sa = oracle.ref_sa(text)
        bwt, primary = oracle.ref_bwt(text)
        assert oracle.ref_check_sa(text, sa)[0] and oracle.ref_check_bwt(text, bwt, primary)[0], name
        large.append({"name": name, "generator": expr, "n": int(len(text)), "text_sha256": digest(text),
                      "sa_sha256": digest(sa.astype("<i4")), "bwt_sha256": digest(bwt), "primary": primary})
        print(name, len(text), primary)
    (HERE / "large.json").write_text(json.dumps({"source": "reference CPU build, cover 128", "cases": large},
                                                indent=1))


if __name__ == "__main__":
    main()
