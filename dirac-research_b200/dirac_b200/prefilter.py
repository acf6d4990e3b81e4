"""The encoder's prefilters over CUDA tensors.

``cwm_filter`` wraps dgpu_cwm_filter, which replaces CWMFilterComponent
(libdirac_encoder/prefilter.cpp:50-125): the reference applies it to each component of an
input picture's working data when the CWM prefilter is selected (seq_compress.cpp:649-651).
``rect_lp_filter`` and ``diag_lp_filter`` wrap dgpu_rect_lp_filter / dgpu_diag_lp_filter, which
replace LPFilter and DiagFilter (prefilter.cpp:141-306, 307-588): the residue prefilters
PictureCompressor::Prefilter applies before the transform (picture_compress.cpp:340-355).
"""
import ctypes

import torch

from . import _lib


def cwm_filter(pic, strength, out=None, stream=None):
    """pic: 2-D int16 CUDA tensor; returns the filtered component (a new tensor unless out)."""
    lib = _lib.load()
    if pic.dtype != torch.int16 or not pic.is_cuda or pic.dim() != 2:
        raise TypeError("expected a 2-D int16 CUDA tensor")
    src = pic.contiguous()
    dst = out if out is not None else torch.empty_like(src)
    h, w = src.shape
    st = stream if stream is not None else torch.cuda.current_stream()
    _lib.check(lib.dgpu_cwm_filter(src.data_ptr(), w, dst.data_ptr(), dst.stride(0), w, h, int(strength),
                                   st.cuda_stream), "dgpu_cwm_filter")
    return dst


def _lp(name, pic, qf, strength, stream=None):
    lib = _lib.load()
    if pic.dtype != torch.int16 or not pic.is_cuda or pic.dim() != 2 or pic.stride(1) != 1:
        raise TypeError("expected a 2-D int16 CUDA tensor with unit column stride")
    h, w = pic.shape
    st = stream if stream is not None else torch.cuda.current_stream()
    _lib.check(getattr(lib, name)(pic.data_ptr(), w, h, pic.stride(0), ctypes.c_float(qf), int(strength), None,
                                  st.cuda_stream), name)
    return pic


def rect_lp_filter(pic, qf, strength, stream=None):
    """RECTLP of a 2-D int16 CUDA tensor, in place (returned)."""
    return _lp("dgpu_rect_lp_filter", pic, qf, strength, stream)


def diag_lp_filter(pic, qf, strength, stream=None):
    """DIAGLP of a 2-D int16 CUDA tensor, in place (returned)."""
    return _lp("dgpu_diag_lp_filter", pic, qf, strength, stream)
