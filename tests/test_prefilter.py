"""The encoder's prefilters.  Centre-weighted median: the oracle's restatement (orc_cwm_filter)
against the reference's CWMFilterComponent (tests/golden/prefilter.npz, and live where
oracle/_ref exists), and the CUDA kernel (dgpu_cwm_filter) against the oracle on every
strength and on sizes that leave no, one or many filtered samples, up to a 1080p component.
RECTLP low-pass: orc_rect_lp_filter against the reference's LPFilter, and the kernels
(dgpu_rect_lp_filter) against the oracle over quality factors and strengths.  DIAGLP low-pass:
orc_diag_lp_filter against the reference's DiagFilter on every bandwidth table, and the kernel
(dgpu_diag_lp_filter) against the oracle up to a 1080p component."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import DIAGLP_CASES, PREFILTER_CASES, RECTLP_CASES  # noqa: E402


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


@pytest.mark.parametrize("k", range(len(RECTLP_CASES)))
def test_oracle_rect_lp_matches_reference_fixture(oracle, golden, k):
    g = golden("prefilter.npz")
    _, _, qf, strength = RECTLP_CASES[k]
    np.testing.assert_array_equal(oracle.rect_lp_filter(g[f"lp{k}_in"], qf, strength), g[f"lp{k}_out"])


def test_oracle_rect_lp_matches_live_reference(oracle):
    from oracle import Reference

    if not Reference.available():
        pytest.skip("reference library not built here")
    ref = Reference()
    rng = np.random.default_rng(14)
    for w, h in [(17, 17), (48, 40), (29, 35)]:
        for qf in (1.0, 4.5, 7.0, 11.0):
            for strength in (0, 2, 6, 10):
                pic = rng.integers(-400, 400, size=(h, w)).astype(np.int16)
                np.testing.assert_array_equal(oracle.rect_lp_filter(pic, qf, strength),
                                              ref.rect_lp_filter(pic, qf, strength))


@pytest.mark.gpu
def test_rect_lp_kernels_match_oracle(gpu, oracle):
    import torch

    from dirac_b200 import _lib

    lib = _lib.load()
    rng = np.random.default_rng(15)
    for w, h, qf, strength in [(17, 17, 7.0, 0), (48, 40, 2.0, 3), (176, 144, 10.0, 5), (1920, 1080, 7.0, 1),
                               (31, 19, 0.5, 10)]:
        pic = rng.integers(-400, 400, size=(h, w)).astype(np.int16)
        t = torch.from_numpy(pic).cuda()
        _lib.check(lib.dgpu_rect_lp_filter(t.data_ptr(), w, h, w, ctypes_float(qf), strength, None,
                                           torch.cuda.current_stream().cuda_stream), "dgpu_rect_lp_filter")
        torch.cuda.synchronize()
        np.testing.assert_array_equal(t.cpu().numpy(), oracle.rect_lp_filter(pic, qf, strength),
                                      err_msg=f"{w}x{h} qf {qf} strength {strength}")


def ctypes_float(x):
    import ctypes

    return ctypes.c_float(x)


def test_rect_lp_rejects_small_components():
    from dirac_b200 import _lib

    assert _lib.load().dgpu_rect_lp_filter(16, 16, 17, 16, 7.0, 0, None, None) == -2


@pytest.mark.parametrize("k", range(len(DIAGLP_CASES)))
def test_oracle_diag_lp_matches_reference_fixture(oracle, golden, k):
    g = golden("prefilter.npz")
    _, _, qf, strength = DIAGLP_CASES[k]
    np.testing.assert_array_equal(oracle.diag_lp_filter(g[f"dg{k}_in"], qf, strength), g[f"dg{k}_out"])


def test_oracle_diag_lp_matches_live_reference(oracle):
    from oracle import Reference

    if not Reference.available():
        pytest.skip("reference library not built here")
    ref = Reference()
    rng = np.random.default_rng(16)
    for w, h in [(7, 7), (20, 13), (48, 40)]:
        for qf in (0.5, 3.0, 4.5, 5.7, 7.0, 10.0):
            for strength in range(11):
                pic = rng.integers(-512, 512, size=(h, w)).astype(np.int16)
                np.testing.assert_array_equal(oracle.diag_lp_filter(pic, qf, strength),
                                              ref.diag_lp_filter(pic, qf, strength))


@pytest.mark.gpu
def test_diag_lp_kernel_matches_oracle(gpu, oracle):
    import torch

    from dirac_b200.prefilter import diag_lp_filter

    rng = np.random.default_rng(17)
    cases = [(w, h, qf, s) for (w, h, qf, s) in DIAGLP_CASES]
    cases += [(176, 144, 5.7, 5), (37, 300, 6.0, 10), (1920, 1080, 4.5, 3), (960, 540, 3.0, 0)]
    for w, h, qf, strength in cases:
        pic = rng.integers(-1024, 1024, size=(h, w)).astype(np.int16)
        t = torch.from_numpy(pic).cuda()
        diag_lp_filter(t, qf, strength)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(t.cpu().numpy(), oracle.diag_lp_filter(pic, qf, strength),
                                      err_msg=f"{w}x{h} qf {qf} strength {strength}")
    # a strided view: the kernel reads and writes through the row pitch
    base = rng.integers(-1024, 1024, size=(64, 80)).astype(np.int16)
    t = torch.from_numpy(base).cuda()
    view = t[3:60, 5:70]
    diag_lp_filter(view, 6.2, 7)
    torch.cuda.synchronize()
    want = base.copy()
    want[3:60, 5:70] = oracle.diag_lp_filter(base[3:60, 5:70], 6.2, 7)
    np.testing.assert_array_equal(t.cpu().numpy(), want)


def test_diag_lp_rejects_small_components():
    from dirac_b200 import _lib

    assert _lib.load().dgpu_diag_lp_filter(16, 6, 17, 6, 7.0, 0, None, None) == -2
