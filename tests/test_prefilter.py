"""The centre-weighted median prefilter: the oracle's restatement (orc_cwm_filter) against the
reference's CWMFilterComponent (tests/golden/prefilter.npz, and live where oracle/_ref
exists), and the CUDA kernel (dgpu_cwm_filter) against the oracle on every strength and on
sizes that leave no, one or many filtered samples, up to a 1080p component."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import PREFILTER_CASES  # noqa: E402


@pytest.mark.parametrize("k", range(len(PREFILTER_CASES)))
def test_oracle_cwm_matches_reference_fixture(oracle, golden, k):
    g = golden("prefilter.npz")
    strength = PREFILTER_CASES[k][2]
    np.testing.assert_array_equal(oracle.cwm_filter(g[f"c{k}_in"], strength), g[f"c{k}_out"])


def test_oracle_cwm_matches_live_reference(oracle):
    from oracle import Reference

    if not Reference.available():
        pytest.skip("reference library not built here")
    ref = Reference()
    rng = np.random.default_rng(12)
    for w, h in [(64, 48), (37, 23), (3, 3), (4, 5)]:
        for strength in range(12):
            pic = rng.integers(-512, 512, size=(h, w)).astype(np.int16)
            np.testing.assert_array_equal(oracle.cwm_filter(pic, strength), ref.cwm_filter(pic, strength))


@pytest.mark.gpu
def test_cwm_kernel_matches_oracle(gpu, oracle):
    import torch

    from dirac_b200.prefilter import cwm_filter

    rng = np.random.default_rng(13)
    cases = [(w, h, s) for (w, h) in [(64, 48), (37, 23), (3, 3), (2, 7), (4, 5), (176, 144)] for s in range(12)]
    cases += [(1920, 1080, 5), (960, 540, 2)]
    for w, h, strength in cases:
        pic = rng.integers(-2048, 2048, size=(h, w)).astype(np.int16)
        got = cwm_filter(torch.from_numpy(pic).cuda(), strength)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(got.cpu().numpy(), oracle.cwm_filter(pic, strength),
                                      err_msg=f"{w}x{h} strength {strength}")
