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


def test_suffix_array_written_from_uint32_without_conversion(tmp_path):
    sa = np.array([5, 3, 1, 0, 4, 2], np.uint32)
    a, b = tmp_path / "a.sa", tmp_path / "b.sa"
    fileio.write_suffix_array(a, sa)
    fileio.write_suffix_array(b, sa.astype(np.int64))
    assert a.read_bytes() == b.read_bytes() == sa.astype("<i4").tobytes()
    fileio.write_suffix_array(a, np.arange(10, dtype=np.uint32), n=4)  # the first n entries only
    assert np.fromfile(a, "<i4").tolist() == [0, 1, 2, 3]


def test_extension_written_and_read_in_chunks(tmp_path, monkeypatch):
    monkeypatch.setattr(fileio, "INT32_LIMIT", 5)
    sa = np.array([9, 2, 7, 0, 4, 8, 1, 6, 3, 5, 10], np.uint32)
    p = tmp_path / "big.sa"
    fileio.write_suffix_array(p, sa, chunk=3)  # 4 chunks, the last one short
    assert np.array_equal(np.fromfile(p, "<u8"), sa.astype(np.uint64))
    assert fileio.read_suffix_array(p, len(sa)).dtype == np.int64
    got = fileio.read_suffix_array(p, len(sa), dtype=np.uint32, chunk=4)
    assert got.dtype == np.uint32 and np.array_equal(got, sa)


def test_uint32_read_of_both_formats_and_of_corrupt_entries(tmp_path):
    p = tmp_path / "x.sa"
    np.array([2, -1, 0], "<i4").tofile(p)  # int32 file: a negative entry reads as out of range
    assert fileio.read_suffix_array(p, 3, dtype=np.uint32).tolist() == [2, 0xFFFFFFFF, 0]
    np.array([1, 1 << 40, 0], "<u8").tofile(p)  # 64-bit file: an entry past 2^32 reads as out of range
    assert fileio.read_suffix_array(p, 3, dtype=np.uint32).tolist() == [1, 0xFFFFFFFF, 0]
    empty = tmp_path / "empty.sa"
    empty.write_bytes(b"")
    assert len(fileio.read_suffix_array(empty, 0)) == 0
    assert len(fileio.read_suffix_array(empty, 0, dtype=np.uint32)) == 0


def test_cli_maps_its_input(tmp_path):
    p = tmp_path / "in.txt"
    p.write_bytes(b"mississippi")
    text = cli._load(p)
    assert isinstance(text, np.memmap) and not text.flags.writeable
    assert bytes(text) == b"mississippi"
    empty = tmp_path / "empty.txt"
    empty.write_bytes(b"")
    assert len(cli._load(empty)) == 0
