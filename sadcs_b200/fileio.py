"""File formats of the reference (src/common/fileio.cpp), plus the extension past its int32 limit.

* Suffix array: n little-endian int32 entries, no header (divsufsort's mksary; fileio.cpp:44-63).
  Extension for texts of more than 2^31 - 1025 bytes (which the reference refuses,
  src/cpu/dcsort.h:21): n little-endian uint64 entries. A reader tells the two apart by the file
  size against the text size (4n or 8n bytes).
* BWT: int32 n, then (n > 0) int32 primary index, then the n bytes (divsufsort's bwt format as one
  block; fileio.cpp:78-125). Extension for n > 2^31 - 1025: int32 -1, int64 n, int64 primary, the
  n bytes.
"""
from __future__ import annotations

import numpy as np

INT32_LIMIT = (1 << 31) - 1025


def write_suffix_array(path, sa: np.ndarray, n: int | None = None) -> None:
    n = len(sa) if n is None else n
    dtype = "<i4" if n <= INT32_LIMIT else "<u8"
    np.ascontiguousarray(sa, dtype=dtype).tofile(path)


def read_suffix_array(path, n: int) -> np.ndarray:
    """The suffix array of a text of n bytes (int32 or, for the extension, uint64 entries)."""
    size = np.memmap(path, dtype=np.uint8, mode="r").size if n else 0
    if size == 4 * n:
        return np.fromfile(path, dtype="<i4").astype(np.int64 if n > INT32_LIMIT else np.int32)
    if size == 8 * n:
        return np.fromfile(path, dtype="<u8").astype(np.int64)
    raise ValueError(f"{path}: {size} bytes is neither 4n nor 8n for n = {n}")


def write_bwt(path, bwt: np.ndarray, primary: int) -> None:
    n = len(bwt)
    with open(path, "wb") as f:
        if n <= INT32_LIMIT:
            f.write(np.int32(n).tobytes())
            if n > 0:
                f.write(np.int32(primary).tobytes())
        else:
            f.write(np.int32(-1).tobytes())
            f.write(np.int64(n).tobytes())
            f.write(np.int64(primary).tobytes())
        f.write(np.ascontiguousarray(bwt, dtype=np.uint8).tobytes())


def read_bwt(path):
    """(bwt bytes, primary index) of a single-block BWT file."""
    data = np.fromfile(path, dtype=np.uint8)
    if data.size < 4:
        raise ValueError(f"{path}: too short for a BWT file")
    n = int(data[:4].view("<i4")[0])
    if n == -1:
        if data.size < 20:
            raise ValueError(f"{path}: truncated extended header")
        n = int(data[4:12].view("<i8")[0])
        primary = int(data[12:20].view("<i8")[0])
        body = data[20:]
    elif n == 0:
        if data.size != 4:
            raise ValueError(f"{path}: an empty BWT has no primary index")
        return np.zeros(0, np.uint8), 0
    elif n > 0:
        if data.size < 8:
            raise ValueError(f"{path}: truncated header")
        primary = int(data[4:8].view("<i4")[0])
        body = data[8:]
    else:
        raise ValueError(f"{path}: negative block size")
    if body.size != n:
        raise ValueError(f"{path}: {body.size} bytes of BWT, header says {n}")
    return body, primary
