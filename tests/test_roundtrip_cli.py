"""The command line end to end on the device: build writes the reference's SA and BWT file formats
(from page-locked outputs the merge writes directly, with the input memory-mapped), check accepts
them and rejects a corrupted one, and a BWT may be written over its own input file, as the
reference's CLI allows (src/cli/main.cpp:358-359). Outputs are compared with the oracle."""
import numpy as np
import pytest

import oracle
from sadcs_b200 import cli, fileio
from sadcs_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_build_then_check(tmp_path):
    text = W.natural_text(300_000, seed=51)
    source = tmp_path / "in.txt"
    text.tofile(source)
    expected = oracle.doubling_sa(text)
    eb, ep = oracle.bwt_from_sa(text, expected)

    assert cli.main(["build", str(source), str(tmp_path / "in.sa")]) == 0
    assert np.array_equal(np.fromfile(tmp_path / "in.sa", "<i4"), expected.astype("<i4"))
    assert cli.main(["build", "--bwt", str(source), str(tmp_path / "in.bwt")]) == 0
    bwt, primary = fileio.read_bwt(tmp_path / "in.bwt")
    assert primary == ep and np.array_equal(bwt, eb)

    assert cli.main(["check", str(source), str(tmp_path / "in.sa")]) == 0
    assert cli.main(["check", "--bwt", str(source), str(tmp_path / "in.bwt")]) == 0
    bad = np.fromfile(tmp_path / "in.sa", "<i4")
    bad[[10, 11]] = bad[[11, 10]]
    bad.tofile(tmp_path / "bad.sa")
    assert cli.main(["check", str(source), str(tmp_path / "bad.sa")]) == 1


def test_bwt_over_its_own_input(tmp_path):
    text = W.random_text(W.SplitMix(52), 70_000, 4)
    path = tmp_path / "text"
    text.tofile(path)
    assert cli.main(["build", "--bwt", str(path), str(path)]) == 0
    eb, ep = oracle.bwt_from_sa(text, oracle.doubling_sa(text))
    bwt, primary = fileio.read_bwt(path)
    assert primary == ep and np.array_equal(bwt, eb)


def test_empty_input(tmp_path):
    source = tmp_path / "empty"
    source.write_bytes(b"")
    assert cli.main(["build", str(source), str(tmp_path / "empty.sa")]) == 0
    assert (tmp_path / "empty.sa").read_bytes() == b""
    assert cli.main(["build", "--bwt", str(source), str(tmp_path / "empty.bwt")]) == 0
    bwt, primary = fileio.read_bwt(tmp_path / "empty.bwt")
    assert len(bwt) == 0 and primary == 0


def test_test_and_selftest_commands(tmp_path):
    """`test` and `test --bwt` build each file and check it against the file itself (text and BWT
    of the same length, the case where a check that freed its device copy of the text too early
    compared the BWT with itself); `selftest` runs the adversarial families through both checks."""
    W.natural_text(300_000, seed=53).tofile(tmp_path / "natural")
    W.random_text(W.SplitMix(54), 50_000, 4).tofile(tmp_path / "dna")
    W.run_text(4096).tofile(tmp_path / "run")
    assert cli.main(["test", str(tmp_path)]) == 0
    assert cli.main(["test", "--bwt", str(tmp_path)]) == 0
    assert cli.main(["selftest"]) == 0


def test_check_rejects_a_bwt_that_is_not_the_texts(tmp_path):
    text = W.natural_text(200_000, seed=55)
    other = W.natural_text(200_000, seed=56)
    source = tmp_path / "in.txt"
    text.tofile(source)
    eb, ep = oracle.bwt_from_sa(other, oracle.doubling_sa(other))
    fileio.write_bwt(tmp_path / "other.bwt", eb, ep)
    assert cli.main(["check", "--bwt", str(source), str(tmp_path / "other.bwt")]) == 1
