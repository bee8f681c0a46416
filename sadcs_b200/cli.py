"""sadcs command line for the GPU path (python -m sadcs_b200 ...).

The reference's commands and flags (src/cli/main.cpp:73-154), its output lines and exit codes
(0 ok, 1 error); the construction always runs on the GPU (cover mod 32; --cover and --threads are
accepted and do not apply, as for the reference's --gpu). Checks run on the GPU too, from host
buffers (sadcs_gpu_check_suffix_array_host / sadcs_gpu_check_bwt_host). Texts past the reference's
int32 limit use the 64-bit file formats of sadcs_b200.fileio. The reference's own CLI also links
unchanged against libsadcs_gpu.so through include/gpusa.h.

  sadcs build|-b [--bwt] <in> <out> [--gpu]
  sadcs check|-c [--bwt] <in> <in.sa|in.bwt>
  sadcs test|-t <in|dir> [--bwt] [--recursive]
  sadcs bench <in|dir> [--bwt] [--runs N] [--context] [--pinned] [--recursive]
  sadcs selftest [--verbose]
"""
from __future__ import annotations

import argparse
import os
import sys
import time
from pathlib import Path

import numpy as np

from . import fileio

EXIT_OK, EXIT_ERROR = 0, 1
MIB = float(1 << 20)


def _mbs(n, seconds):
    return n / MIB / seconds if seconds > 0 else 0.0


def _files(path: Path, recursive: bool):
    if path.is_dir():
        it = path.rglob("*") if recursive else path.iterdir()
        return sorted(p for p in it if p.is_file())
    return [path]


def _load(path) -> np.ndarray:
    """A regular input file memory-mapped read-only: no copy into process memory; the
    construction's upload reads the pages straight from the mapping. Anything else (a pipe) is
    read in full."""
    if not os.path.isfile(path):
        return np.fromfile(path, dtype=np.uint8)
    if os.path.getsize(path) == 0:
        return np.zeros(0, np.uint8)
    return np.memmap(path, dtype=np.uint8, mode="r")


def _pinned_outputs(n: int, want_sa: bool, want_bwt: bool):
    """Page-locked output buffers (the construction's merge writes them directly, with no separate
    download), or None where page-locked memory is not available."""
    import sadcs_b200 as sa

    if n == 0:
        return None, None, []
    owned = []
    try:
        out_sa = out_bwt = None
        if want_sa:
            owned.append(sa.allocate_pinned(4 * n))
            out_sa = owned[-1].view(np.uint32)
        if want_bwt:
            owned.append(sa.allocate_pinned(n))
            out_bwt = owned[-1]
        return out_sa, out_bwt, owned
    except MemoryError:
        for buffer in owned:
            sa.free_pinned(buffer)
        return None, None, []


def _gpu_error(e) -> int:
    import sadcs_b200 as sa

    kind = {sa.GpuStatus.Unavailable: "unavailable", sa.GpuStatus.NotEnoughMemory: "out of memory"}.get(
        getattr(e, "status", None), "failed")
    print(f"sadcs: GPU {kind}: {e}")
    return EXIT_ERROR


def check_sa(text: np.ndarray, sa_array: np.ndarray):
    """(ok, first failing SA index, reason): the reference checker's fast mode, on the device."""
    import sadcs_b200 as sa

    return sa.check_suffix_array(text, np.ascontiguousarray(sa_array, dtype=np.uint32))


def check_bwt(text: np.ndarray, bwt: np.ndarray, primary: int):
    """(ok, first text position where the inverse differs): the reference's BWT check, on the device."""
    import sadcs_b200 as sa

    return sa.check_bwt(text, bwt, primary)


def cmd_build(a) -> int:
    import sadcs_b200 as sa

    if len(a.paths) != 2:
        print(__doc__)
        return EXIT_ERROR
    text = _load(a.paths[0])
    n = len(text)
    stats = sa.Stats()
    out_sa, out_bwt, owned = _pinned_outputs(n, not a.bwt, a.bwt)
    try:
        start = time.perf_counter()
        try:
            suffixes, bwt, primary = sa.build(text, want_sa=not a.bwt, want_bwt=a.bwt, stats=stats, out_sa=out_sa,
                                              out_bwt=out_bwt)
        except sa.GpuError as e:
            return _gpu_error(e)
        seconds = time.perf_counter() - start
        if a.bwt:
            fileio.write_bwt(a.paths[1], bwt, primary)
        else:
            fileio.write_suffix_array(a.paths[1], suffixes)
    finally:
        for buffer in owned:
            sa.free_pinned(buffer)
    print(f"{a.paths[0]} -> {a.paths[1]}: {n} bytes, GPU, {seconds:.3f}s ({_mbs(n, seconds):.1f} MB/s), peak device "
          f"memory {stats.device_bytes / MIB:.1f} MiB ({stats.device_bytes / max(n, 1):.2f} bytes per input byte)")
    return EXIT_OK


def cmd_check(a) -> int:
    if len(a.paths) != 2:
        print(__doc__)
        return EXIT_ERROR
    text = _load(a.paths[0])
    n = len(text)
    start = time.perf_counter()
    if a.bwt:
        try:
            bwt, primary = fileio.read_bwt(a.paths[1])
        except ValueError:
            print(f"sadcs: cannot read '{a.paths[1]}' as a single-block BWT file")
            return EXIT_ERROR
        if len(bwt) != n:
            print(f"sadcs: '{a.paths[1]}' has {len(bwt)} bytes of BWT, but '{a.paths[0]}' has {n} bytes")
            return EXIT_ERROR
        ok, index = check_bwt(text, bwt, primary)
        seconds = time.perf_counter() - start
        if not ok:
            print(f"sadcs: BWT check FAILED (primary index {primary}): inverse BWT differs from the text, index {index}")
            return EXIT_ERROR
        print(f"{a.paths[1]}: BWT OK ({n} bytes, primary index {primary}, {seconds:.3f}s)")
        return EXIT_OK
    try:
        sa_array = fileio.read_suffix_array(a.paths[1], n, dtype=np.uint32)
    except ValueError:
        print(f"sadcs: cannot read '{a.paths[1]}' as a suffix array")
        return EXIT_ERROR
    ok, index, reason = check_sa(text, sa_array)
    seconds = time.perf_counter() - start
    if not ok:
        print(f"sadcs: check FAILED at SA[{index}]: {reason}")
        return EXIT_ERROR
    print(f"{a.paths[1]}: suffix array OK ({n} entries, {seconds:.3f}s)")
    return EXIT_OK


def _test_one(path, bwt_mode: bool):
    import sadcs_b200 as sa

    text = _load(path)
    n = len(text)
    stats = sa.Stats()
    start = time.perf_counter()
    suffixes, bwt, primary = sa.build(text, want_sa=not bwt_mode, want_bwt=bwt_mode, stats=stats)
    build = time.perf_counter() - start
    start = time.perf_counter()
    ok = check_bwt(text, bwt, primary)[0] if bwt_mode else check_sa(text, suffixes)[0]
    return n, build, time.perf_counter() - start, stats, ok


def cmd_test(a) -> int:
    import sadcs_b200 as sa

    if len(a.paths) != 1:
        print(__doc__)
        return EXIT_ERROR
    files = _files(Path(a.paths[0]), a.recursive)
    width = max([5] + [len(str(f)) for f in files])
    print(f"{a.paths[0]}: {len(files)} files, {'BWT' if a.bwt else 'suffix array'}, GPU (times in seconds)")
    print(f"{'file':<{width}} {'bytes':>12} {'gpu':>8} {'MB/s':>8} {'peak/n':>6} {'check':>8}")
    passed = 0
    for f in files:
        try:
            n, build, check, stats, ok = _test_one(f, a.bwt)
        except sa.GpuError as e:
            return _gpu_error(e)
        passed += ok
        print(f"{str(f):<{width}} {n:>12} {build:>8.3f} {_mbs(n, build):>8.1f} {stats.device_bytes / max(n, 1):>6.2f} "
              f"{check:>8.3f}  {'OK' if ok else 'FAILED'}")
    print(f"{passed}/{len(files)} OK")
    return EXIT_OK if passed == len(files) else EXIT_ERROR


def cmd_bench(a) -> int:
    import sadcs_b200 as sa

    if len(a.paths) != 1:
        print(__doc__)
        return EXIT_ERROR
    files = _files(Path(a.paths[0]), a.recursive)
    try:
        device = sa.query_device()
    except sa.GpuError as e:
        return _gpu_error(e)
    print(f"{a.paths[0]}: {len(files)} file{'s' if len(files) != 1 else ''}, GPU {device['name']}, "
          f"{'BWT' if a.bwt else 'suffix array'}, best of {a.runs} runs{', context reused' if a.context else ''}"
          f"{', pinned host buffers' if a.pinned else ''} (times in ms)")
    width = max([5] + [len(f.name) for f in files])
    print(f"{'file':<{width}} {'bytes':>12} {'setup':>7} {'upload':>7} {'rank':>7} {'class':>7} {'merge':>7} "
          f"{'down':>7} {'total':>8} {'MB/s':>7} {'peak/n':>6}")
    for f in files:
        text = _load(f)
        n = len(text)
        ctx = sa.Context(n) if a.context else None
        source = text
        if a.pinned:
            source = sa.allocate_pinned(n)
            source[:] = text
        best, best_stats = None, None
        try:
            for run in range(a.runs + 1):
                stats = sa.Stats()
                start = time.perf_counter()
                sa.build(source, want_sa=not a.bwt, want_bwt=a.bwt, context=ctx, stats=stats)
                seconds = time.perf_counter() - start
                if run > 0 and (best is None or seconds < best):
                    best, best_stats = seconds, stats
        except sa.GpuError as e:
            return _gpu_error(e)
        finally:
            if ctx:
                ctx.close()
            if a.pinned:
                sa.free_pinned(source)
        s = best_stats
        print(f"{f.name:<{width}} {n:>12} {s.setup_seconds * 1e3:>7.1f} {s.upload_seconds * 1e3:>7.1f} "
              f"{s.ranking_seconds * 1e3:>7.1f} {s.class_sort_seconds * 1e3:>7.1f} {s.merge_seconds * 1e3:>7.1f} "
              f"{s.download_seconds * 1e3:>7.1f} {best * 1e3:>8.1f} {_mbs(n, best):>7.1f} "
              f"{s.device_bytes / max(n, 1):>6.2f}")
    return EXIT_OK


def cmd_selftest(a) -> int:
    """GPU constructions of the reference selftest's adversarial families, each verified by the GPU
    suffix-array checker and the BWT inversion check."""
    import sadcs_b200 as sa
    from . import workloads as W

    rng = W.SplitMix(3)
    cases = [(w.decode() or '""', np.frombuffer(w, np.uint8)) for w in (b"a", b"banana", b"mississippi")]
    cases += [(f"run of a, n={n}", W.run_text(n)) for n in range(1, 81)]
    cases += [(f"random sigma=2, n={n}", W.random_text(rng, n, 2)) for n in range(1, 81)]
    cases += [(f"period {p}", W.periodic_text(rng, 5000, p)) for p in (1, 2, 3, 5, 7, 31, 32, 33, 63, 64, 65, 1000)]
    cases += [("fibonacci", W.fibonacci_text(5000)), ("fibonacci 0/1", W.fibonacci_text(5000, 0, 1)),
              ("thue-morse", W.thue_morse_text(4096)), ("zeros", np.zeros(1000, np.uint8))]
    for sigma in (1, 2, 4, 26, 256):
        cases += [(f"random sigma={sigma} #{i}", W.random_text(rng, 1 + int(rng.below(20000)[0]), sigma))
                  for i in range(10)]
    failures = 0
    for name, text in cases:
        try:
            suffixes, bwt, primary = sa.build(text)
            ok = check_sa(text, suffixes)[0] and check_bwt(text, bwt, primary)[0]
        except sa.GpuError as e:
            return _gpu_error(e)
        if not ok:
            failures += 1
            print(f"  FAIL {name}")
        elif a.verbose:
            print(f"  ok   {name} (n={len(text)})")
    print(f"selftest: {len(cases) - failures} of {len(cases)} cases passed")
    return EXIT_OK if failures == 0 else EXIT_ERROR


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if not argv:
        print(__doc__)
        return EXIT_ERROR
    command, rest = argv[0], argv[1:]
    p = argparse.ArgumentParser(prog="sadcs", add_help=False)
    p.add_argument("paths", nargs="*")
    p.add_argument("--bwt", action="store_true")
    p.add_argument("--gpu", action="store_true")
    p.add_argument("--cover", type=int, default=128)
    p.add_argument("--threads", type=int, default=0)
    p.add_argument("--runs", type=int, default=5)
    p.add_argument("--context", action="store_true")
    p.add_argument("--pinned", action="store_true")
    p.add_argument("--recursive", action="store_true")
    p.add_argument("--verbose", action="store_true")
    p.add_argument("--lowmem", action="store_true")
    p.add_argument("--naive", action="store_true")
    try:
        a = p.parse_args(rest)
    except SystemExit:
        return EXIT_ERROR
    if a.cover not in (64, 128, 256):
        print("sadcs: --cover must be 64, 128 or 256")
        return EXIT_ERROR
    handlers = {"build": cmd_build, "-b": cmd_build, "check": cmd_check, "-c": cmd_check, "test": cmd_test,
                "-t": cmd_test, "bench": cmd_bench, "selftest": cmd_selftest}
    if command not in handlers:
        print(__doc__)
        return EXIT_ERROR
    return handlers[command](a)


if __name__ == "__main__":
    sys.exit(main())
