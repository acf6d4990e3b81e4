"""Host-side behaviour of the decoder entry points, without a GPU: sizing, and the argument
checks that reject a call before anything is queued (dgpu_dequantise_batch refuses a coded
band whose quantiser index is outside 0..119, as the reference decoder does,
band_codec_template.h:250-258; dgpu_decoder_* refuse invalid parameters)."""
import ctypes

import numpy as np
import pytest


def lib():
    from dirac_b200 import _lib

    return _lib.load()


def params(**kw):
    from dirac_b200.decoder import decoder_params

    cfg = dict(cformat=2, width=1920, height=1080, luma_depth=8, chroma_depth=8, wlt_depth=4, mv_precision=2,
               xblen=16, yblen=16, xbsep=12, ybsep=12)
    cfg.update(kw)
    return decoder_params(cfg)


def test_decoder_device_bytes():
    from dirac_b200.decoder import device_bytes

    one = device_bytes(params(), 1)
    eight = device_bytes(params(), 8)
    # per 1080p 4:2:0 slot: planes (2 B), coefficients padded to 1920 x 1088 (4 B), upconverted planes (8 B)
    slot = (eight - one) / 7
    samples = 1920 * 1080 * 1.5
    assert samples * 14 <= slot <= samples * 14 * 1.02
    assert device_bytes(params(luma_depth=10, chroma_depth=10), 8) == eight


@pytest.mark.parametrize("bad", [dict(cformat=3), dict(wlt_depth=0), dict(wlt_depth=7), dict(luma_depth=7),
                                 dict(width=8), dict(xbsep=20)])
def test_decoder_rejects_bad_parameters(bad):
    from dirac_b200.decoder import device_bytes

    with pytest.raises(ValueError):
        device_bytes(params(**bad), 4)
    handle = ctypes.c_void_p()
    p = params(**bad)
    assert lib().dgpu_decoder_create(ctypes.byref(p), 4, None, ctypes.byref(handle)) == -1
    assert not handle.value


def _dequantise_call(band_qidx, band_skip, depth=1, ncb=None, cw=8, ch=8):
    from dirac_b200 import _lib

    nb = 3 * depth + 1
    ncb = ncb if ncb is not None else [1, 1] * nb
    dummy = ctypes.c_void_p(16)  # never dereferenced: the call is refused before any launch
    return lib().dgpu_dequantise_batch(
        1, _lib.int_array([0]), _lib.int_array([depth]), _lib.ptr_array([dummy.value]), _lib.ptr_array([dummy.value]),
        _lib.int_array([cw]), _lib.int_array([ch]), _lib.int_array(ncb), _lib.int_array(band_qidx),
        _lib.int_array(band_skip), dummy, None)


def test_dequantise_refuses_before_launch():
    assert _dequantise_call([120, 0, 0, 0], [0, 0, 0, 0]) == -1        # quantiser index above 119
    assert _dequantise_call([-1, 0, 0, 0], [0, 0, 0, 0]) == -1         # negative index
    assert _dequantise_call([0, 0, 0, 0], [0, 0, 0, 0], cw=7) == -1    # not a multiple of 2^depth
    assert _dequantise_call([0, 0, 0, 0], [0, 0, 0, 0], ncb=[0, 1] * 4) == -1   # no code blocks
    assert _dequantise_call([0] * 4, [0] * 4, depth=9, ncb=[1, 1] * 28) == -1   # depth beyond 8


def test_decoder_null_handles():
    L = lib()
    assert L.dgpu_decoder_destroy(None) == -1
    assert L.dgpu_decoder_release(None, 0) == -1
    assert L.dgpu_decoder_decode(None, None) == -1
    assert L.dgpu_decoder_item_bytes(None, 0, 0, 0) == 0
    buf = np.zeros(4, np.uint8)
    assert L.dgpu_decoder_read(None, 0, 0, 0, buf.ctypes.data, 4, 1) == -1


def test_decode_bytes_model():
    """The decoding leg's algorithmic bytes: 8 B per coefficient for the dequantisation, the
    inverse transform as the encoder's, OBMC ADD with the clip for inter pictures (the clip
    alone for intra ones) and one upconversion per reference picture used."""
    from dirac_b200.roofline import decode_bytes, dwt_bytes

    params = dict(cformat=2, width=64, height=32, luma_depth=8, chroma_depth=8, wlt_depth=2)
    infos = [dict(intra=1, num_refs=0, ref1=-1, ref2=-1),
             dict(intra=0, num_refs=1, ref1=0, ref2=-1),
             dict(intra=0, num_refs=2, ref1=0, ref2=1)]
    b = decode_bytes(params, infos)
    coeffs = 64 * 32 + 2 * 32 * 16
    samples = coeffs  # sizes are multiples of 4: no padding
    assert b["dequantisation"] == 3 * 8 * coeffs
    assert b["dwt_inverse"] == 3 * (dwt_bytes(64, 32, 2) + 2 * dwt_bytes(32, 16, 2))
    assert b["mc_add_clip"] == samples * 4 + samples * (4 + 8) + samples * (4 + 16)
    assert b["upconvert"] == 2 * samples * 10
    # pictures decoded from int16 indices read 2 B instead of 4 per coefficient
    b16 = decode_bytes(params, infos, int16_pictures=2)
    assert b16["dequantisation"] == 3 * 8 * coeffs - 2 * 2 * coeffs
    assert {k: v for k, v in b16.items() if k != "dequantisation"} == \
        {k: v for k, v in b.items() if k != "dequantisation"}
