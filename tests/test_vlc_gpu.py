"""The variable-length coefficient coder on the device (dgpu_code_bands_vlc) against the host
one (dgpu_code_bands_vlc_host), which is byte-equal to the reference's BandVLC /
IntraDCBandVLC (tests/test_band_coder.py): the same bytes, band byte counts and exact bit
counts, on index arrays that stress the codes (zeros, large values, near-even signs, whole
zero code blocks), with one code block per band and several, skipped bands and code blocks,
and on several components of different sizes coded together."""
import numpy as np
import pytest

from test_band_coder import _adversarial_indices

pytestmark = pytest.mark.gpu

KINDS = ["zero", "huge", "signs", "even", "sparse", "blocks", "stripes"]


def both(depth, qs, bands, ncbs, cbss):
    import torch

    from dirac_b200.entropy import code_bands, code_bands_vlc_device

    want = code_bands([0] * len(qs), depth, qs, bands, ncbs, cbss, vlc=True)
    got = code_bands_vlc_device(depth, [torch.from_numpy(q).cuda() for q in qs], bands, ncbs, cbss)
    return want, got


def cb_flags(q, depth, ncb, rng, p_skip):
    """Code-block skip flags set at random with probability p_skip (the coder codes what it
    is told)."""
    ch, cw = q.shape
    flags = []
    for b in range(1, 3 * depth + 2):
        xn, yn = ncb[b - 1]
        flags += [int(rng.random() < p_skip) for _ in range(xn * yn)]
    return np.array(flags, np.uint8)


@pytest.mark.parametrize("kind", KINDS)
def test_device_vlc_equals_host_vlc(gpu, kind):
    depth = 4
    rng = np.random.default_rng(sum(map(ord, kind)) + 7)
    q = _adversarial_indices(kind, rng)
    for ncb in (np.ones((3 * depth + 1, 2), np.int32),
                np.array([[1, 1]] * 4 + [[2, 2]] * 3 + [[4, 3]] * 3 + [[3, 4]] * 3, np.int32)[::-1].copy()):
        for p_skip in (0.0, 0.3):
            bands = np.zeros((3 * depth + 1, 3), np.int32)
            bands[rng.integers(0, 3 * depth + 1, size=2), 1] = 1 if p_skip else 0  # two skipped bands
            cbs = cb_flags(q, depth, ncb, rng, p_skip)
            (wd, wper, wbits), (gd, gper, gbits) = both(depth, [q], [bands], [ncb], [cbs])
            np.testing.assert_array_equal(gper[0], wper[0], err_msg=kind)
            np.testing.assert_array_equal(gbits[0], wbits[0], err_msg=kind)
            assert gd.tobytes() == wd.tobytes(), kind


def test_device_vlc_several_components(gpu):
    """Three components of a 4:2:0 picture (different sizes and depths' code-block layouts)
    in one call: the data component by component, each from the DC band down."""
    from dirac_b200 import quant

    rng = np.random.default_rng(99)
    depth = 4
    shapes = [(144, 176), (80, 96), (80, 96)]  # padded to 16 for depth 4
    qs = [(rng.standard_cauchy(size=s) * 3).clip(-3000, 3000).astype(np.int32) for s in shapes]
    ncb = quant.code_blocks(depth, 176, 144).reshape(-1, 2)
    bands = [np.zeros((3 * depth + 1, 3), np.int32) for _ in qs]
    bands[1][5, 1] = 1
    cbss = [cb_flags(q, depth, ncb, rng, 0.2) for q in qs]
    (wd, wper, wbits), (gd, gper, gbits) = both(depth, qs, bands, [ncb] * 3, cbss)
    for c in range(3):
        np.testing.assert_array_equal(gper[c], wper[c])
        np.testing.assert_array_equal(gbits[c], wbits[c])
    assert gd.tobytes() == wd.tobytes()
