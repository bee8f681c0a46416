"""This library against the reference's own CUDA build on the same GPU (oracle/_ref/libsadcs_ref_gpu.so:
the reference's gpusa.cu compiled unchanged for sm_100a). Both must give the same SA, BWT and
primary index on the same seeded texts; the CPU oracle is the third party to every comparison.
Skipped where the reference build is absent."""
import numpy as np
import pytest

import oracle
import sadcs_b200 as sa
from sadcs_b200 import workloads as W

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_gpu_available(), reason="reference CUDA build not present")]


def _cases():
    rng = W.SplitMix(77)
    return [
        ("empty", np.zeros(0, np.uint8)),
        ("one", np.array([7], np.uint8)),
        ("zeros", np.zeros(1000, np.uint8)),
        ("abc", W.random_text(rng, 5000, 3)),
        ("fibonacci", W.fibonacci_text(20000)),
        ("thue-morse", W.thue_morse_text(65536)),
        ("uniform-1m", W.uniform_bytes(1 << 20, seed=5)),
        ("natural-4m", W.natural_text(4 << 20, seed=6)),
        ("genome-4m", W.genome_text(4 << 20, seed=7)),
    ]


@pytest.fixture(scope="module")
def ref_context():
    ctx = oracle.RefGpuContext(4 << 20)
    yield ctx
    ctx.close()


@pytest.mark.parametrize("name,text", _cases(), ids=[c[0] for c in _cases()])
def test_same_as_reference_gpu(name, text, ref_context):
    ours_sa, ours_bwt, ours_primary = sa.build(text)
    ref_sa, _ = ref_context.suffix_array(text)
    ref_bwt, ref_primary, _ = ref_context.bwt(text)
    assert np.array_equal(ours_sa.astype(np.int64), ref_sa.astype(np.int64)), name
    assert ours_primary == ref_primary, name
    assert np.array_equal(ours_bwt, ref_bwt), name
    if len(text) <= (1 << 20):
        ok, where = oracle.check_sa(text, ours_sa.astype(np.uint32))
        assert ok, (name, where)
