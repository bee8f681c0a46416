"""File formats (the reference's, and the 64-bit extension) and the CLI's argument handling, CPU only."""
import numpy as np
import pytest

from sadcs_b200 import cli, fileio


def test_suffix_array_file_int32(tmp_path):
    sa = np.array([5, 3, 1, 0, 4, 2], np.int32)
    p = tmp_path / "x.sa"
    fileio.write_suffix_array(p, sa)
    assert p.stat().st_size == 4 * len(sa)
    assert np.array_equal(np.fromfile(p, "<i4"), sa)  # divsufsort's mksary layout
    assert np.array_equal(fileio.read_suffix_array(p, 6), sa)
    with pytest.raises(ValueError):
        fileio.read_suffix_array(p, 7)


def test_bwt_file_layout(tmp_path):
    p = tmp_path / "x.bwt"
    fileio.write_bwt(p, np.frombuffer(b"annb$aa"[:6], np.uint8), 4)
    raw = p.read_bytes()
    assert raw[:4] == (6).to_bytes(4, "little") and raw[4:8] == (4).to_bytes(4, "little") and len(raw) == 14
    bwt, primary = fileio.read_bwt(p)
    assert primary == 4 and bytes(bwt) == b"annb$a"
    fileio.write_bwt(p, np.zeros(0, np.uint8), 0)
    assert p.read_bytes() == (0).to_bytes(4, "little")
    assert fileio.read_bwt(p)[1] == 0


def test_bwt_file_extension_header(tmp_path, monkeypatch):
    monkeypatch.setattr(fileio, "INT32_LIMIT", 3)
    p = tmp_path / "big.bwt"
    fileio.write_bwt(p, np.frombuffer(b"abcde", np.uint8), 2)
    raw = p.read_bytes()
    assert raw[:4] == (0xFFFFFFFF).to_bytes(4, "little") and len(raw) == 20 + 5
    bwt, primary = fileio.read_bwt(p)
    assert bytes(bwt) == b"abcde" and primary == 2
    fileio.write_suffix_array(p, np.arange(5))
    assert p.stat().st_size == 40 and fileio.read_suffix_array(p, 5).tolist() == [0, 1, 2, 3, 4]


def test_cli_rejects_bad_usage(capsys):
    assert cli.main([]) == 1
    assert cli.main(["frobnicate"]) == 1
    assert cli.main(["build", "only-one-path"]) == 1
    assert cli.main(["build", "a", "b", "--cover", "7"]) == 1
    assert "cover must be" in capsys.readouterr().out
