"""The encoder's centre-weighted median prefilter over CUDA tensors.

``cwm_filter`` wraps dgpu_cwm_filter, which replaces CWMFilterComponent
(libdirac_encoder/prefilter.cpp:50-125): the reference applies it to each component of an
input picture's working data when the CWM prefilter is selected (seq_compress.cpp:649-651).
"""
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
