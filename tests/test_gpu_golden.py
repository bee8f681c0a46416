"""This library against the reference CPU build's own outputs at the benchmark sizes: every case of
tests/golden/large.json (SHA-256 of the int32 SA and of the BWT bytes, made by the reference's
buildSuffixArray / buildBwt, cover 128) is built on the device and its digests compared, among
them the 8 MiB i.i.d. uniform text of seed 1 the reference's CPU-runnable benchmark is quoted on.
The 256 MiB natural-language-like text is compared with the reference's own CUDA build on the same
GPU (oracle/_ref/libsadcs_ref_gpu.so), entry by entry."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
import sadcs_b200 as sa
from sadcs_b200 import workloads as W

pytestmark = pytest.mark.gpu

LARGE = json.loads((Path(__file__).parent / "golden" / "large.json").read_text())["cases"]


def _digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("case", LARGE, ids=[c["name"] for c in LARGE])
def test_reference_digests(case):
    text = eval(case["generator"], {"W": W})
    assert len(text) == case["n"] and _digest(text) == case["text_sha256"], "generator drifted"
    suffixes, bwt, primary = sa.build(text)
    assert _digest(suffixes.astype("<i4")) == case["sa_sha256"]
    assert primary == case["primary"] and _digest(bwt) == case["bwt_sha256"]
    # the reference's int32 entry points give the same arrays
    assert _digest(sa.suffix_array(text).astype("<i4")) == case["sa_sha256"]
    b2, p2 = sa.bwt(text)
    assert p2 == case["primary"] and _digest(b2) == case["bwt_sha256"]


@pytest.mark.skipif(not oracle.ref_gpu_available(), reason="reference CUDA build not present")
def test_natural_256m_same_as_reference_gpu():
    import torch

    text = W.natural_text(256 << 20, seed=2)
    n = len(text)
    ctx = oracle.RefGpuContext(n)
    try:
        ref_sa, _ = ctx.suffix_array(text)
        ref_bwt, ref_primary, _ = ctx.bwt(text)
    finally:
        ctx.close()
    d_text = torch.from_numpy(text).cuda()
    d_sa = torch.empty(n, dtype=torch.int32, device="cuda")
    d_bwt = torch.empty(n, dtype=torch.uint8, device="cuda")
    primary = sa.build_device(d_text.data_ptr(), n, d_sa.data_ptr(), d_bwt.data_ptr())
    torch.cuda.synchronize()
    assert primary == ref_primary
    assert torch.equal(d_sa, torch.from_numpy(ref_sa).cuda())
    assert torch.equal(d_bwt, torch.from_numpy(ref_bwt).cuda())
