"""Host-side mirror of the reference's WaveletTransform interface over device tensors.

Reference: ``WaveletTransform(int d = 4, WltFilter f = DAUB9_7)`` and
``Transform(const Direction d, PicArray& pic_data, CoeffArray& coeff_data)``
(libdirac_common/wavelet_utils.h:686-728).  Here a PicArray is an int16 CUDA tensor of shape
(h, w) and a CoeffArray an int32 CUDA tensor of shape (ch, cw), both possibly row-strided.
"""
import torch

from . import _lib

DD9_7, LEGALL5_3, DD13_7, HAAR0, HAAR1, FIDELITY, DAUB9_7 = range(7)
FILTER_NAMES = ["DD9_7", "LEGALL5_3", "DD13_7", "HAAR0", "HAAR1", "FIDELITY", "DAUB9_7"]
FORWARD, BACKWARD = 0, 1


def padded_size(w, h, depth):
    """Coefficient-array size for a w x h component (Picture::InitWltData, picture.cpp:201-219)."""
    mul = 1 << depth
    return (w + mul - 1) // mul * mul, (h + mul - 1) // mul * mul


def _stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def _check_tensor(t, dtype, name):
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype or t.dim() != 2 or t.stride(1) != 1:
        raise ValueError(f"{name} must be a 2-D {dtype} tensor with unit column stride")


class WaveletTransform:
    """Forward / inverse Dirac wavelet transform on the GPU (no CPU fallback)."""

    def __init__(self, depth=4, filt=DAUB9_7):
        self.lib = _lib.load()
        self.depth = depth
        self.filter = filt

    def Transform(self, direction, pic_data, coeff_data, scratch=None, stream=None):
        _check_tensor(pic_data, torch.int16, "pic_data")
        _check_tensor(coeff_data, torch.int32, "coeff_data")
        h, w = pic_data.shape
        ch, cw = coeff_data.shape
        sptr, sbytes = (None, 0)
        if scratch is not None:
            sptr, sbytes = scratch.data_ptr(), scratch.numel() * scratch.element_size()
        rc = self.lib.dgpu_wavelet_transform(
            direction, self.filter, self.depth,
            pic_data.data_ptr(), w, h, pic_data.stride(0),
            coeff_data.data_ptr(), cw, ch, coeff_data.stride(0),
            sptr, sbytes, _stream_ptr(stream))
        _lib.check(rc, "dgpu_wavelet_transform")

    def scratch_bytes(self, cw, ch):
        return self.lib.dgpu_dwt_scratch_bytes(cw, ch, self.depth)


def transform_batch(direction, items, scratch=None, stream=None):
    """Several transforms in one launch per level.

    items: list of (filter, depth, pic int16 tensor, coeff int32 tensor)."""
    lib = _lib.load()
    n = len(items)
    filt = _lib.int_array([it[0] for it in items])
    depth = _lib.int_array([it[1] for it in items])
    pics = [it[2] for it in items]
    coeffs = [it[3] for it in items]
    for p in pics:
        _check_tensor(p, torch.int16, "pic")
    for c in coeffs:
        _check_tensor(c, torch.int32, "coeff")
    sptr, sbytes = (None, 0)
    if scratch is not None:
        sptr, sbytes = scratch.data_ptr(), scratch.numel() * scratch.element_size()
    rc = lib.dgpu_wavelet_transform_batch(
        direction, n, filt, depth,
        _lib.ptr_array([p.data_ptr() for p in pics]),
        _lib.int_array([p.shape[1] for p in pics]),
        _lib.int_array([p.shape[0] for p in pics]),
        _lib.int_array([p.stride(0) for p in pics]),
        _lib.ptr_array([c.data_ptr() for c in coeffs]),
        _lib.int_array([c.shape[1] for c in coeffs]),
        _lib.int_array([c.shape[0] for c in coeffs]),
        _lib.int_array([c.stride(0) for c in coeffs]),
        sptr, sbytes, _stream_ptr(stream))
    _lib.check(rc, "dgpu_wavelet_transform_batch")
