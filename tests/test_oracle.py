"""The CPU oracle (oracle/dirac_oracle.c) pinned against the reference codec.

Golden fixtures in tests/golden were produced by running the reference's own C++
(tests/golden/make_golden.py).  Where oracle/_ref is built, the oracle is additionally
checked differentially against the live reference on fresh seeded inputs.
"""
import numpy as np
import pytest

from oracle import Reference


def test_dwt_golden_forward_and_backward(oracle, golden):
    g = golden("dwt.npz")
    metas = [k[:-5] for k in g.files if k.endswith("_meta")]
    assert len(metas) == 21
    for key in metas:
        filt, depth, w, h, cw, ch = (int(v) for v in g[key + "_meta"])
        coeff = oracle.dwt_forward(filt, depth, g[key + "_pic"], cw, ch)
        np.testing.assert_array_equal(coeff, g[key + "_coeff"], err_msg=key)
        back = oracle.dwt_backward(filt, depth, g[key + "_noisy"], w, h)
        np.testing.assert_array_equal(back, g[key + "_back"], err_msg=key)


def test_upconvert_golden(oracle, golden):
    g = golden("convert.npz")
    for k in range(3):
        w, h, bd = (int(v) for v in g[f"up{k}_meta"])
        np.testing.assert_array_equal(oracle.upconvert(g[f"up{k}_pic"], bd), g[f"up{k}_out"])


def test_downconvert_golden(oracle, golden):
    g = golden("convert.npz")
    for k in range(3):
        np.testing.assert_array_equal(oracle.downconvert(g[f"down{k}_pic"]), g[f"down{k}_out"])


def ramp(w, h):
    """The reference unit test's picture: (((i-j) % 13) * 1024) / 13 with C semantics
    (unit_tests/wavelet_utils_test.cpp:50-58)."""
    j, i = np.mgrid[0:h, 0:w]
    d = i - j
    m = np.fmod(d, 13)  # C remainder keeps the dividend's sign
    v = m * 1024
    return (np.sign(v) * (np.abs(v) // 13)).astype(np.int16)  # C division truncates


@pytest.mark.parametrize("filt", range(8))
def test_transform_invertibility_ramp(oracle, filt):
    """Restates unit_tests/wavelet_utils_test.cpp:84-105: 512x512 ramp, depth 1, every
    WltFilter value (FIDELITY and filterNK fall through to DAUB9_7): forward then
    backward returns the input."""
    pic = ramp(512, 512)
    coeff = oracle.dwt_forward(filt, 1, pic)
    np.testing.assert_array_equal(oracle.dwt_backward(filt, 1, coeff, 512, 512), pic)


@pytest.mark.parametrize("filt", range(7))
def test_invertibility_deep(oracle, filt):
    rng = np.random.default_rng(filt)
    pic = rng.integers(-512, 512, size=(77, 131)).astype(np.int16)
    for depth in (2, 4):
        coeff = oracle.dwt_forward(filt, depth, pic)
        np.testing.assert_array_equal(oracle.dwt_backward(filt, depth, coeff, 131, 77), pic)


def test_rejects_undefined_sizes(oracle):
    # a DD filter level side below 6 reads outside the region in the reference
    with pytest.raises(ValueError):
        oracle.dwt_forward(0, 3, np.zeros((16, 16), np.int16))
    with pytest.raises(ValueError):
        oracle.downconvert(np.zeros((22, 40), np.int16))


needs_ref = pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built here")


@needs_ref
@pytest.mark.parametrize("filt", range(7))
def test_dwt_matches_live_reference(oracle, filt):
    ref = Reference()
    rng = np.random.default_rng(100 + filt)
    for (w, h, depth) in [(352, 288, 4), (176, 144, 5), (101, 67, 3), (720, 576, 5)]:
        pic = rng.integers(-128, 128, size=(h, w)).astype(np.int16)
        c_ref = ref.dwt_forward(filt, depth, pic)
        np.testing.assert_array_equal(oracle.dwt_forward(filt, depth, pic), c_ref)
        noisy = (c_ref + rng.integers(-20, 21, size=c_ref.shape)).astype(np.int32)
        np.testing.assert_array_equal(oracle.dwt_backward(filt, depth, noisy, w, h),
                                      ref.dwt_backward(filt, depth, noisy, w, h))


@needs_ref
def test_convert_matches_live_reference(oracle):
    ref = Reference()
    rng = np.random.default_rng(3)
    for (w, h, bd) in [(352, 288, 8), (176, 144, 10), (960, 540, 8)]:
        pic = rng.integers(-(1 << (bd - 1)), 1 << (bd - 1), size=(h, w)).astype(np.int16)
        np.testing.assert_array_equal(oracle.upconvert(pic, bd), ref.upconvert(pic, bd))
        np.testing.assert_array_equal(oracle.downconvert(pic), ref.downconvert(pic))
