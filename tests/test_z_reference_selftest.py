"""The reference's own selftest (src/cli/selftest.cpp, unchanged) compiled against this library's
C++ shim (include/gpusa.h over libsadcs_gpu.so) by `make -C oracle ref-on-b200`: its CPU cases, its
checker's planted errors, and its GPU cases (src/cli/selftest.cpp:432-606: every GPU suffix array,
in-place BWT and sample ranking compared with the reference's CPU construction, a reused context
and its over-capacity refusal), all run by the reference's own harness. The binary is built where
the reference sources are; the test is skipped where it is absent."""
import re
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

BINARY = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "sadcs_on_b200"


def test_reference_selftest_passes_on_this_library():
    if not BINARY.exists():
        pytest.skip("oracle/_ref/sadcs_on_b200 is not built (needs the reference sources)")
    run = subprocess.run([str(BINARY), "selftest"], capture_output=True, text=True, timeout=1200)
    out = run.stdout + run.stderr
    assert "GPU vs. CPU on" in out, out[-2000:]  # the GPU cases ran, not skipped
    passed = re.search(r"selftest: (\d+) of (\d+) cases passed", out)
    assert passed and passed.group(1) == passed.group(2), out[-2000:]
    assert run.returncode == 0, out[-2000:]
