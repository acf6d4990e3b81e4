"""The 3840x2160 4:2:2 10-bit workload (48 rectangles moving at up to 64 px/frame): motion
estimation over the reference's depth-7 pyramid (pixel_match.cpp:94-95 at this size), quarter-pel
refinement and mode decision of a B picture, OBMC 16x16 at separation 12 (SUBTRACT and ADD)
with those motion data, upconversion of a 10-bit reference, and Deslauriers-Dubuc (9,7) depth-5
transforms of every component.  tests/golden/uhd.npz holds the reference's own results as
CRC-32s (tests/golden/make_golden.py); the oracle is checked against them on the CPU and the
CUDA path on the GPU, both bit for bit."""
import os
import sys
import zlib

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import UHD_LAMBDA, uhd_inputs  # noqa: E402


def crc(a):
    return zlib.crc32(np.ascontiguousarray(a).tobytes())


@pytest.fixture(scope="module")
def uhd():
    return uhd_inputs()


def test_uhd_inputs_match_fixture(uhd, golden):
    f, _ = uhd
    g = golden("uhd.npz")
    np.testing.assert_array_equal(np.array([[crc(c) for c in fr] for fr in f], np.uint32), g["in"])


def test_oracle_uhd_motion_estimation_and_compensation_match_reference(uhd, oracle, golden):
    f, bp = uhd
    g = golden("uhd.npz")
    assert oracle.me_depth(3840, 2160) == 7
    me = oracle.motion_estimate(1, f[1], f[0], f[2], bp, UHD_LAMBDA, 3, luma_depth=10)
    for k, v in me.items():
        assert crc(v) == int(g["me_" + k]), k
    for aos in (0, 1):
        res = oracle.motion_compensate(aos, 1, f[1], f[0], f[2], bp, me["mv"][0], me["mv"][1], me["mode"], me["dc"],
                                       me["split"], luma_depth=10, chroma_depth=10)
        np.testing.assert_array_equal([crc(c) for c in res], g[f"mc{aos}"], err_msg=f"aos {aos}")


def test_oracle_uhd_transform_and_upconversion_match_reference(uhd, oracle, golden):
    f, _ = uhd
    g = golden("uhd.npz")
    np.testing.assert_array_equal([crc(oracle.upconvert(c, 10)) for c in f[0]], g["up"])
    for c in range(3):
        co = oracle.dwt_forward(0, 5, f[1][c])
        assert crc(co) == int(g["dwt_fwd"][c]), c
        assert crc(oracle.dwt_backward(0, 5, co, f[1][c].shape[1], f[1][c].shape[0])) == int(g["dwt_back"][c]), c


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.gpu
def test_gpu_uhd_motion_estimation_and_compensation(gpu, uhd, golden):
    """Device estimation of the B picture equals the reference's (vectors, float costs, modes, DC
    values, splits, superblock costs); device OBMC with those data equals the reference's."""
    f, bp = uhd
    g = golden("uhd.npz")
    bpg = gpu.BlockParams(bp.precision, bp.xblen, bp.yblen, bp.xbsep, bp.ybsep, bp.xnum_sb, bp.ynum_sb)
    me = gpu.MotionEstimator(bpg, 1, 10).Estimate([_dev(p) for p in f[1]], [_dev(p) for p in f[0]],
                                                  [_dev(p) for p in f[2]], UHD_LAMBDA, 3)
    got = {k: v.cpu().numpy() for k, v in me.items()}
    for k, v in got.items():
        assert crc(v) == int(g["me_" + k]), k
    ups1 = [gpu.upconvert(_dev(r), 10) for r in f[0]]
    ups2 = [gpu.upconvert(_dev(r), 10) for r in f[2]]
    np.testing.assert_array_equal([crc(u.cpu().numpy()) for u in ups1], g["up"])
    mc = gpu.MotionCompensator(bpg, 1)
    for aos in (0, 1):
        p = [_dev(x) for x in f[1]]
        mc.CompensatePicture(aos, me["mv"][0].contiguous(), me["mv"][1].contiguous(), me["mode"], me["dc"],
                             me["split"], p, ups1, ups2)
        np.testing.assert_array_equal([crc(x.cpu().numpy()) for x in p], g[f"mc{aos}"], err_msg=f"aos {aos}")


@pytest.mark.gpu
def test_gpu_uhd_transforms(gpu, uhd, golden):
    import torch

    f, _ = uhd
    g = golden("uhd.npz")
    wt = gpu.WaveletTransform(5, gpu.DD9_7)
    for c in range(3):
        pic = _dev(f[1][c])
        h, w = f[1][c].shape
        cw, ch = gpu.padded_size(w, h, 5)
        co = torch.zeros((ch, cw), dtype=torch.int32, device="cuda")
        wt.Transform(gpu.FORWARD, pic, co)
        assert crc(co.cpu().numpy()) == int(g["dwt_fwd"][c]), c
        back = torch.zeros_like(pic)
        wt.Transform(gpu.BACKWARD, back, co)
        assert crc(back.cpu().numpy()) == int(g["dwt_back"][c]), c
