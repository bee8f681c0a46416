"""The final merge's tiling (sadcs_b200/csrc/merge.cuh, planTileWindows and the rows of the level
above), restated in numpy: for any interleaving of the 7 sorted class lists, every tile's window set
fits the fixed shared-memory capacity G*R + 6*(G-1) + 1, the windows hold every element the tile
outputs, and an element's output index (the windows' total start plus its rank among them) is its
position in the merged order. The kernel has no overflow path, so this bound is what keeps it in
bounds whatever the text. Also the bound the overlapped download of the last level relies on: no
output below a tile's window base comes from that tile or a later one (its C++ form, tileOutputBound,
through tests/plan_harness.cu)."""
import numpy as np
import pytest

CLASSES = 7
G = 32


def merged_positions(lists):
    """(values, list of each, index within its list) of all elements in merged (value) order."""
    values = np.concatenate(lists)
    which = np.concatenate([np.full(len(l), b) for b, l in enumerate(lists)])
    index = np.concatenate([np.arange(len(l)) for l in lists])
    order = np.argsort(values, kind="stable")
    return values[order], which[order], index[order]


def rows_of_level_above(lists, R):
    """Rows from merging the splitters (every G-th element of each list): for every R-th element s
    of their merged order, s's list and c_b = the splitters of list b smaller than s; then the end."""
    splitters = [l[::G] for l in lists]
    values, which, index = merged_positions(splitters)
    rows = []
    for g in range(0, len(values), R):
        v, l = values[g], which[g]
        c = [int(index[g]) if b == l else int(np.searchsorted(splitters[b], v)) for b in range(CLASSES)]
        rows.append((int(l), c, v))
    rows.append((None, [len(s) for s in splitters], None))
    return rows


def windows(lo, hi, lens):
    """planTileWindows: [w_b, e_b) of each list for the tile between rows lo and hi."""
    w, e = [], []
    for b in range(CLASSES):
        if lo[0] is None:
            wb = 0
        elif b == lo[0]:
            wb = lo[1][b] * G
        else:
            wb = 0 if lo[1][b] == 0 else (lo[1][b] - 1) * G + 1
        if hi[0] is None:
            eb = lens[b]
        elif b == hi[0]:
            eb = hi[1][b] * G + 1
        else:
            eb = min(lens[b], hi[1][b] * G)
        wb = min(wb, lens[b])
        eb = max(min(eb, lens[b]), wb)
        w.append(wb)
        e.append(eb)
    return w, e


def check_tiling(lists, R):
    cap = G * R + 6 * (G - 1) + 1
    lens = [len(l) for l in lists]
    values = np.sort(np.concatenate(lists))
    rows = rows_of_level_above(lists, R)
    written = np.zeros(len(values), dtype=np.int64)
    starts = []  # (window base, first output) of every tile
    for t in range(len(rows) - 1):
        lo, hi = rows[t], rows[t + 1]
        w, e = windows(lo, hi, lens)
        size = sum(e[b] - w[b] for b in range(CLASSES))
        assert size <= cap, (t, size, cap)
        base = sum(w)
        window = np.sort(np.concatenate([lists[b][w[b]:e[b]] for b in range(CLASSES)]))
        # elements before a window are smaller than s_lo, elements after it not smaller than s_hi
        for b in range(CLASSES):
            if lo[0] is not None:
                assert np.all(lists[b][:w[b]] < lo[2])
            if hi[0] is not None:
                assert np.all(lists[b][e[b]:] >= hi[2])
        # the tile writes the window elements from s_lo up to s_hi, at base + rank
        first = 0 if lo[0] is None else int(np.searchsorted(window, lo[2]))
        last = len(window) if hi[0] is None else int(np.searchsorted(window, hi[2]))
        for r in range(first, last):
            pos = base + r
            assert values[pos] == window[r]
            written[pos] += 1
        starts.append((base, base + first))
    assert np.all(written == 1)
    # Tiles own consecutive output ranges in tile order, each starting at or above its window base:
    # once tiles [0, t) are done, every output below tile t's base is final.
    for t, (base, first_out) in enumerate(starts):
        assert base <= first_out, (t, base, first_out)
        assert t == 0 or starts[t - 1][1] <= first_out
    return rows, starts


def class_sized_lists(rng, n, assign):
    """7 sorted lists of distinct values with the class sizes of a mod-32 cover (7,6,5,5,4,3,2 of 32),
    the values drawn by `assign` (which list each merged position goes to)."""
    sizes = np.array([7, 6, 5, 5, 4, 3, 2]) * n // 32
    owner = assign(rng, sizes)
    return [np.flatnonzero(owner == b).astype(np.int64) for b in range(CLASSES)]


def random_assign(rng, sizes):
    owner = np.repeat(np.arange(CLASSES), sizes)
    rng.shuffle(owner)
    return owner


def block_assign(rng, sizes):
    """Long runs of one list at a time: windows of the other lists stay short, one list long."""
    runs = []
    left = sizes.copy()
    while left.sum():
        b = rng.choice(np.flatnonzero(left))
        k = min(left[b], int(rng.integers(1, 5000)))
        runs.append(np.full(k, b))
        left[b] -= k
    return np.concatenate(runs)


def staircase_assign(rng, sizes):
    """Each list's elements all together, in list order: every tile but the boundary ones reads one
    list."""
    return np.repeat(np.arange(CLASSES), sizes)


def comb_assign(rng, sizes):
    """Runs of exactly G - 1 of a list, rotating through the lists: splitters fall just inside runs,
    the windows' (G - 1) slack at both ends is used as much as the data allows."""
    left = sizes.copy()
    runs = []
    b = 0
    while left.sum():
        if left[b]:
            k = min(left[b], G - 1)
            runs.append(np.full(k, b))
            left[b] -= k
        b = (b + 1) % CLASSES
    return np.concatenate(runs)


@pytest.mark.parametrize("R", [26, 40, 80])  # 40: records of several code words; 80: of one
@pytest.mark.parametrize("assign", [random_assign, block_assign, staircase_assign, comb_assign])
def test_tiles_fit_and_cover_the_output(R, assign):
    rng = np.random.default_rng(11)
    for n in (2000, 65536, 200000):
        check_tiling(class_sized_lists(rng, n, assign), R)


def test_tiles_with_empty_and_tiny_lists():
    rng = np.random.default_rng(5)
    for sizes in ([0, 0, 0, 0, 0, 0, 5000], [1, 0, 3, 0, 2, 0, 40000], [G * 41, 1, 1, 1, 1, 1, 1]):
        owner = np.repeat(np.arange(CLASSES), sizes)
        rng.shuffle(owner)
        lists = [np.flatnonzero(owner == b).astype(np.int64) for b in range(CLASSES)]
        for R in (40, 80):
            check_tiling(lists, R)


def test_tile_output_bound_matches_the_library():
    """tileOutputBound (merge.cuh, host code) gives each tile's window base, as restated above."""
    from tests.test_memory_plan import harness

    lib = harness()
    import ctypes

    lib.plan_tile_bound.restype = ctypes.c_uint64
    lib.plan_tile_bound.argtypes = [ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]
    rng = np.random.default_rng(8)
    for assign in (random_assign, block_assign, comb_assign):
        for n in (3000, 100000):
            lists = class_sized_lists(rng, n, assign)
            lens = [len(l) for l in lists]
            start = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint32)
            rows, starts = check_tiling(lists, 40)
            for t in range(len(rows) - 1):
                lo = rows[t]
                row = np.array([0xFFFFFFFF if lo[0] is None else lo[0], *lo[1]], dtype=np.uint32)
                got = lib.plan_tile_bound(row.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                          start.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
                assert got == starts[t][0], (t, got, starts[t][0])
