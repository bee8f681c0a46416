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

import os

import numpy as np

INT32_LIMIT = (1 << 31) - 1025
CHUNK = 1 << 24  # entries converted at a time for the 64-bit format (128 MiB of uint64)


def write_suffix_array(path, sa: np.ndarray, n: int | None = None, chunk: int = CHUNK) -> None:
    """Writes the first n entries of sa. int32 entries are written from the array itself when it
    holds 32-bit integers (no converted copy); the 64-bit extension converts chunk entries at a
    time, so a 3 GiB text's suffix array never needs a 24 GiB uint64 copy."""
    a = np.asarray(sa)
    n = len(a) if n is None else n
    a = a[:n]
    if n <= INT32_LIMIT:
        if a.dtype in (np.int32, np.uint32) and a.dtype.byteorder in "=<|" and a.flags.c_contiguous:
            a.view("<i4").tofile(path)  # entries of a suffix array of n <= INT32_LIMIT are below 2^31
        else:
            np.ascontiguousarray(a, dtype="<i4").tofile(path)
        return
    with open(path, "wb") as f:
        for start in range(0, n, chunk):
            np.ascontiguousarray(a[start:start + chunk], dtype="<u8").tofile(f)


def read_suffix_array(path, n: int, dtype=None, chunk: int = CHUNK) -> np.ndarray:
    """The suffix array of a text of n bytes (int32 or, for the extension, uint64 entries).

    By default int32 entries come back as int32 (int64 past INT32_LIMIT) and uint64 ones as int64.
    dtype=np.uint32 reads either format into one uint32 array (what the device checker takes), the
    64-bit one chunk entries at a time; an entry that does not fit (a corrupt file) becomes
    0xFFFFFFFF, which the checker reports as out of range."""
    size = os.path.getsize(path) if n else 0
    if size == 4 * n:
        a = np.fromfile(path, dtype="<i4") if n else np.zeros(0, "<i4")
        if dtype is not None and np.dtype(dtype) == np.uint32:
            return a.view(np.uint32)
        return a.astype(np.int64 if n > INT32_LIMIT else np.int32, copy=False)
    if size == 8 * n:
        if dtype is not None and np.dtype(dtype) == np.uint32:
            out = np.empty(n, np.uint32)
            with open(path, "rb") as f:
                for start in range(0, n, chunk):
                    part = np.fromfile(f, dtype="<u8", count=min(chunk, n - start))
                    out[start:start + len(part)] = np.minimum(part, 0xFFFFFFFF)
            return out
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
        np.ascontiguousarray(bwt, dtype=np.uint8).tofile(f)


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
