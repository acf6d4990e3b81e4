"""The drop-in: the reference codec built with the bodies of its hot-path methods replaced by
calls into libdiracgpu (oracle/dropin/dropin_shims.cpp: WaveletTransform::Transform,
MotionCompensator::CompensatePicture, PictureCompressor::PixelME / SubPixelME /
ModeDecisionME / SelectQuantisers), driven through its unchanged public APIs.  Encoding through
dirac_encoder_* (stock adaptive entropy factors, arithmetic or variable-length coefficient
coding) gives byte for byte the stock reference encoder's bitstream; decoding that bitstream
through dirac_decoder_* (its inverse transforms and motion compensation on the GPU) gives the
stock encoder's locally decoded pictures (arithmetic-coded streams: the reference decoder
takes variable-length coefficient data in intra pictures only).  The stock bitstreams' lengths and CRC-32s, and the
pictures' CRC-32s, are the reference's own (tests/golden/adaptive.npz, hd1080.npz)."""
import os
import sys
import zlib

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import ENCODE_CASES, encode_inputs, hd_inputs  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dropin(gpu):
    from oracle import DROPIN_SO, Reference

    if not Reference.available(DROPIN_SO):
        pytest.skip("oracle/_ref/libdirac_dropin.so not built (needs the reference sources at build time)")
    return DROPIN_SO


def _crcs(frames):
    return np.array([[zlib.crc32(np.ascontiguousarray(p).tobytes()) for p in f] for f in frames], np.uint32)


def _encode_decode(gpu, path, seq, cfg, decode=True):
    from oracle import reference_decode, reference_encode_stream

    lib = gpu.load()
    n0 = lib.dgpu_launch_count()
    rec, ptype, stream = reference_encode_stream(cfg, seq, freeze=False, path=path)
    n1 = lib.dgpu_launch_count()
    assert n1 > n0, "the drop-in encoder did not reach the GPU path"
    if not decode:
        return rec, ptype, bytes(stream), None
    dec = reference_decode(stream, cfg["width"], cfg["height"], cfg["cformat"], len(seq), path=path)
    n2 = lib.dgpu_launch_count()
    assert n2 > n1, "the drop-in decoder did not reach the GPU path"
    assert all(f is not None for f in dec)
    return rec, ptype, bytes(stream), dec


@pytest.mark.parametrize("vlc", [0, 1], ids=["arith", "vlc"])
@pytest.mark.parametrize("case", ENCODE_CASES, ids=[c[0] for c in ENCODE_CASES])
def test_dropin_bitstream_equals_stock_reference(gpu, golden, dropin, case, vlc):
    seq, cfg = encode_inputs(case)
    # the reference decoder decodes variable-length coefficient data of intra pictures only
    # ("VLC codes ... supported for Intra frames only"), so the -use_vlc streams are checked
    # on the encoder side: bytes and locally decoded pictures
    rec, ptype, stream, dec = _encode_decode(gpu, dropin, seq, dict(cfg, use_vlc=vlc), decode=not vlc)
    g = golden("adaptive.npz")
    key = case[0] + ("_vlc" if vlc else "")
    assert len(stream) == int(g[key + "_stream_bytes"])
    assert zlib.crc32(stream) == int(g[key + "_stream_crc"])
    np.testing.assert_array_equal(ptype, g[key + "_ptype"])
    np.testing.assert_array_equal(_crcs(rec), g[key + "_crc"])
    if dec is not None:
        np.testing.assert_array_equal(_crcs(dec), g[key + "_crc"])


def test_dropin_hd1080_bitstream_equals_stock_reference(gpu, golden, dropin):
    """The 1080p workload (HD1080P50 preset, QF 7, DAUB9_7 / DD9_7, OBMC 16/12, quarter-pel):
    the first 10 frames of the bench's sequence through the stock API on the drop-in build."""
    seq, cfg = hd_inputs()
    rec, ptype, stream, dec = _encode_decode(gpu, dropin, seq, cfg)
    g = golden("hd1080.npz")
    assert len(stream) == int(g["adaptive_stream_bytes"])
    assert zlib.crc32(stream) == int(g["adaptive_stream_crc"])
    np.testing.assert_array_equal(ptype, g["adaptive_ptype"])
    np.testing.assert_array_equal(_crcs(rec), g["adaptive_crc"])
    np.testing.assert_array_equal(_crcs(dec), g["adaptive_decode_crc"])
