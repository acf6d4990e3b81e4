"""Host-side arithmetic coding of quantised subbands and the entropy-correction factors.

``code_bands`` wraps dgpu_code_bands_host: the bytes the reference's band coders write
(CompCompressor::Compress, libdirac_encoder/comp_compress.cpp:64-140) from the signed quantised
indices the device path produces.  ``EntropyCorrector`` wraps dgpu_entropy_*: the reference's
EntropyCorrector (libdirac_common/common.cpp:57-151), whose factors, adapted from the coded
byte counts, make the device encoder choose quantisers as the stock reference encoder does.
No GPU is used here.
"""
import numpy as np

from . import _lib


def code_bands(intra, depth, qindex, bands, ncb, cb_skip, vlc=False):
    """Codes components (vlc: the variable-length form, dgpu_code_bands_vlc_host).  qindex: list
    of int32 [ch][cw] arrays (int16 ones go to dgpu_code_bands_host16, arithmetic form only);
    bands: per component
    [3*depth+1][>=2] (quantiser index, skip, ...), e.g. DGPU_ENC_BANDS; ncb: per component the
    [nb][2] code-block counts; cb_skip: per component the flags.  intra / depth: one value or
    one per component.  Returns (data bytes, band_bytes per component), and with vlc the exact
    bit counts per component as a third item."""
    lib = _lib.load()
    n = len(qindex)
    intra = list(intra) if hasattr(intra, "__len__") else [int(intra)] * n
    depth = list(depth) if hasattr(depth, "__len__") else [int(depth)] * n
    idx16 = not vlc and all(np.asarray(a).dtype == np.int16 for a in qindex)
    q = [np.ascontiguousarray(a, np.int16 if idx16 else np.int32) for a in qindex]
    b = [np.asarray(x, np.int32).reshape(3 * d + 1, -1) for x, d in zip(bands, depth)]
    bq = np.ascontiguousarray(np.concatenate([x[:, 0] for x in b]), np.int32)
    bs = np.ascontiguousarray(np.concatenate([x[:, 1] for x in b]), np.int32)
    nc = np.ascontiguousarray(np.concatenate([np.asarray(x, np.int32).ravel() for x in ncb]), np.int32)
    cbs = np.ascontiguousarray(np.concatenate([np.asarray(x, np.uint8).ravel() for x in cb_skip]), np.uint8)
    nbytes = np.zeros(bq.size, np.int32)
    nbits = np.zeros(bq.size, np.int64)
    cap = sum(a.size for a in q) * 4 + 4096
    while True:
        out = np.zeros(cap, np.uint8)
        args = [n, _lib.int_array(intra), _lib.int_array(depth), _lib.ptr_array([a.ctypes.data for a in q]),
                _lib.int_array([a.shape[1] for a in q]), _lib.int_array([a.shape[0] for a in q]),
                nc.ctypes.data_as(_lib.P_int), bq.ctypes.data_as(_lib.P_int), bs.ctypes.data_as(_lib.P_int),
                cbs.ctypes.data, out.ctypes.data, cap, nbytes.ctypes.data_as(_lib.P_int)]
        if vlc:
            rc = lib.dgpu_code_bands_vlc_host(*args, nbits.ctypes.data)
        else:
            rc = (lib.dgpu_code_bands_host16 if idx16 else lib.dgpu_code_bands_host)(*args)
        if rc == -2:
            cap = int(nbytes.sum()) + 16
            continue
        _lib.check(rc, "dgpu_code_bands_host")
        break
    per, k = [], 0
    for d in depth:
        per.append(nbytes[k:k + 3 * d + 1].copy())
        k += 3 * d + 1
    if vlc:
        bits_per, k = [], 0
        for d in depth:
            bits_per.append(nbits[k:k + 3 * d + 1].copy())
            k += 3 * d + 1
        return out[:int(nbytes.sum())].copy(), per, bits_per
    return out[:int(nbytes.sum())].copy(), per


def code_bands_vlc_device(depth, qindex, bands, ncb, cb_skip, stream=None):
    """dgpu_code_bands_vlc: the variable-length form of code_bands from CUDA int32 tensors
    (qindex: list of [ch][cw] tensors); bands, ncb, cb_skip as for code_bands.  Returns (data
    bytes, band_bytes per component, exact bit counts per component)."""
    import torch

    lib = _lib.load()
    n = len(qindex)
    depth = list(depth) if hasattr(depth, "__len__") else [int(depth)] * n
    for t in qindex:
        if t.dtype != torch.int32 or not t.is_cuda or not t.is_contiguous():
            raise TypeError("expected contiguous int32 CUDA tensors")
    b = [np.asarray(x, np.int32).reshape(3 * d + 1, -1) for x, d in zip(bands, depth)]
    bs = np.ascontiguousarray(np.concatenate([x[:, 1] for x in b]), np.int32)
    nc = np.ascontiguousarray(np.concatenate([np.asarray(x, np.int32).ravel() for x in ncb]), np.int32)
    cbs = np.ascontiguousarray(np.concatenate([np.asarray(x, np.uint8).ravel() for x in cb_skip]), np.uint8)
    nbytes = np.zeros(bs.size, np.int32)
    nbits = np.zeros(bs.size, np.int64)
    st = (stream or torch.cuda.current_stream()).cuda_stream
    args = [n, _lib.int_array(depth), _lib.ptr_array([t.data_ptr() for t in qindex]),
            _lib.int_array([t.shape[1] for t in qindex]), _lib.int_array([t.shape[0] for t in qindex]),
            nc.ctypes.data, bs.ctypes.data, cbs.ctypes.data]
    _lib.check(lib.dgpu_code_bands_vlc(*args, None, 0, nbytes.ctypes.data, nbits.ctypes.data, None, 0, st),
               "dgpu_code_bands_vlc")
    total = int(nbytes.sum())
    out = torch.empty(max(4, (total + 3) // 4 * 4), dtype=torch.uint8, device="cuda")
    _lib.check(lib.dgpu_code_bands_vlc(*args, out.data_ptr(), out.numel(), nbytes.ctypes.data, nbits.ctypes.data,
                                       None, 0, st), "dgpu_code_bands_vlc")
    data = out[:total].cpu().numpy()
    per, bits_per, k = [], [], 0
    for d in depth:
        per.append(nbytes[k:k + 3 * d + 1].copy())
        bits_per.append(nbits[k:k + 3 * d + 1].copy())
        k += 3 * d + 1
    return data, per, bits_per


def decode_bands(depth, shapes, band_skip, ncb, data, band_bytes, vlc=False):
    """dgpu_decode_bands_host: components' signed quantised indices from their coded band data.
    depth: one value or one per component; shapes: (ch, cw) per component; band_skip, ncb and
    band_bytes per component (band-list order); data: the bands' bytes (per component, DC band
    first).  Returns (list of int32 [ch][cw] indices, list of code-block flag arrays)."""
    lib = _lib.load()
    n = len(shapes)
    depth = list(depth) if hasattr(depth, "__len__") else [int(depth)] * n
    q = [np.zeros(s, np.int32) for s in shapes]
    bs = np.ascontiguousarray(np.concatenate([np.asarray(x, np.int32).ravel() for x in band_skip]), np.int32)
    nc = np.ascontiguousarray(np.concatenate([np.asarray(x, np.int32).ravel() for x in ncb]), np.int32)
    bb = np.ascontiguousarray(np.concatenate([np.asarray(x, np.int32).ravel() for x in band_bytes]), np.int32)
    d = np.ascontiguousarray(data, np.uint8) if len(data) else np.zeros(1, np.uint8)
    ncbt = [int((np.asarray(x).reshape(-1, 2)[:, 0] * np.asarray(x).reshape(-1, 2)[:, 1]).sum()) for x in ncb]
    cbs = np.zeros(sum(ncbt), np.uint8)
    _lib.check(lib.dgpu_decode_bands_host(
        n, _lib.int_array(depth), _lib.int_array([s[1] for s in shapes]), _lib.int_array([s[0] for s in shapes]),
        nc.ctypes.data_as(_lib.P_int), bs.ctypes.data_as(_lib.P_int), d.ctypes.data, len(data),
        bb.ctypes.data_as(_lib.P_int),
        int(bool(vlc)), _lib.ptr_array([a.ctypes.data for a in q]), cbs.ctypes.data), "dgpu_decode_bands_host")
    flags, k = [], 0
    for t in ncbt:
        flags.append(cbs[k:k + t].copy())
        k += t
    return q, flags


class EntropyCorrector:
    """The reference's EntropyCorrector for one sequence (transform depth fixed)."""

    def __init__(self, depth):
        self.lib = _lib.load()
        self.depth = depth
        self.nb = 3 * depth + 1
        self.state = np.zeros(9 * self.nb, np.float32)
        _lib.check(self.lib.dgpu_entropy_init(depth, self.state.ctypes.data), "dgpu_entropy_init")

    def factors(self, intra, is_b):
        """[3][3*depth+1] factors for a picture (the ecf argument of code_next)."""
        out = np.zeros((3, self.nb), np.float32)
        _lib.check(self.lib.dgpu_entropy_factors(self.depth, self.state.ctypes.data, int(bool(intra)), int(bool(is_b)),
                                                 out.ctypes.data), "dgpu_entropy_factors")
        return out

    def update(self, intra, is_b, comp, band_skip, est_bits, band_bytes):
        sk = np.ascontiguousarray(band_skip, np.int32)
        eb = np.ascontiguousarray(est_bits, np.int32)
        bb = np.ascontiguousarray(band_bytes, np.int32)
        _lib.check(self.lib.dgpu_entropy_update(self.depth, self.state.ctypes.data, int(bool(intra)), int(bool(is_b)),
                                                comp, sk.ctypes.data_as(_lib.P_int), eb.ctypes.data_as(_lib.P_int),
                                                bb.ctypes.data_as(_lib.P_int)), "dgpu_entropy_update")
