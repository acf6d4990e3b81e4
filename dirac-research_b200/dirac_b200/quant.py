"""Host-side mirror of the reference's residue quantisation over device tensors.

References: PictureCompressor::SelectQuantisers / QuantChooser
(libdirac_encoder/picture_compress.cpp:603-709, quant_chooser.cpp:62-362),
CompCompressor::Compress and the band coders' quantise-and-reconstruct
(comp_compress.cpp:64-156, band_codec_template.h:53-174), CoeffArray::SetBandWeights
(wavelet_utils.cpp:192-395), EncoderParams::SetUsualCodeBlocks (common.cpp:488-510).
"""
import ctypes

import numpy as np
import torch

from . import _lib


def band_weights(filt, depth, cw, ch, comp, cformat, cpd, cpd_scale=1.0, field_coding=False):
    out = np.zeros(3 * depth + 1, np.float64)
    rc = _lib.load().dgpu_band_weights(filt, depth, cw, ch, comp, cformat, ctypes.c_float(cpd),
                                       ctypes.c_float(cpd_scale), int(field_coding),
                                       out.ctypes.data_as(ctypes.c_void_p))
    _lib.check(rc, "dgpu_band_weights")
    return out


def code_blocks(depth, luma_w, luma_h, spatial_partition=True):
    out = np.zeros(2 * (3 * depth + 1), np.int32)
    rc = _lib.load().dgpu_code_blocks(depth, luma_w, luma_h, int(spatial_partition),
                                      out.ctypes.data_as(ctypes.c_void_p))
    _lib.check(rc, "dgpu_code_blocks")
    return out


def code_residue(components, stream=None, qout=None):
    """Quantiser choice and in-place quantisation of a batch of transformed components.

    components: list of dicts with keys coeff (int32 CUDA tensor, dense), intra (bool),
    depth, lambda_, band_wt (per band, float), band_ecf (per band), band_ncb (2 per band).
    qout: optional list of int32 CUDA tensors shaped like coeff for the quantised indices.
    Returns per component dicts: qidx, skip, bits (numpy), cb_skip (numpy uint8)."""
    lib = _lib.load()
    n = len(components)
    wt = np.concatenate([np.asarray(c["band_wt"], np.float32) for c in components])
    ecf = np.concatenate([np.asarray(c["band_ecf"], np.float32) for c in components])
    ncb = np.concatenate([np.asarray(c["band_ncb"], np.int32) for c in components])
    nb = len(wt)
    qidx = np.zeros(nb, np.int32)
    skip = np.zeros(nb, np.int32)
    bits = np.zeros(nb, np.int32)
    ncbt = int(np.sum(ncb[0::2] * ncb[1::2]))
    cbs = np.zeros(max(ncbt, 1), np.uint8)
    for c in components:
        t = c["coeff"]
        if not (t.is_cuda and t.dtype == torch.int32 and t.is_contiguous()):
            raise ValueError("coeff must be a dense int32 CUDA tensor")
    lam = np.asarray([c["lambda_"] for c in components], np.float32)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = lib.dgpu_code_residue_batch(
        n, _lib.int_array([int(bool(c["intra"])) for c in components]),
        _lib.int_array([c["depth"] for c in components]),
        _lib.ptr_array([c["coeff"].data_ptr() for c in components]),
        _lib.int_array([c["coeff"].shape[1] for c in components]),
        _lib.int_array([c["coeff"].shape[0] for c in components]), P(lam), P(wt), P(ecf),
        ncb.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), qidx.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
        skip.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), bits.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
        P(cbs), _lib.ptr_array([q.data_ptr() for q in qout]) if qout is not None else None, None, 0,
        (stream if stream is not None else torch.cuda.current_stream()).cuda_stream)
    _lib.check(rc, "dgpu_code_residue_batch")
    out, b0, k0 = [], 0, 0
    for c in components:
        m = 3 * c["depth"] + 1
        nc = int(np.sum(ncb[2 * b0:2 * (b0 + m):2] * ncb[2 * b0 + 1:2 * (b0 + m):2]))
        out.append({"qidx": qidx[b0:b0 + m].copy(), "skip": skip[b0:b0 + m].copy(), "bits": bits[b0:b0 + m].copy(),
                    "cb_skip": cbs[k0:k0 + nc].copy()})
        b0 += m
        k0 += nc
    return out
