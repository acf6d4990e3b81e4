"""Host-side mirror of the reference decoder's picture decoding over the library's device decoder.

``SequenceDecoder`` wraps the dgpu_decoder_* entry points.  The caller does what stays
serial host code in the reference (parsing and entropy decoding: PictureDecompressor's
DecompressMVData and the band decoders' symbol decoding, libdirac_decoder/picture_decompress.cpp
and band_codec_template.h) and hands each picture's signed quantised indices, band
quantisers and skip flags, code-block skip flags and motion data to ``decode``; the device
decoder dequantises, inverse-transforms, motion-compensates and clips
(PictureDecompressor::Decompress, picture_decompress.cpp:73-212) and converts to output
samples on ``read(..., OUTPUT)`` (set_frame_component, dirac_parser.cpp:159-226).

``dequantise`` exposes the dequantisation stage alone (dgpu_dequantise_batch).
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import BlockParams
from .encoder import COEFF, OUTPUT, RECON


class DecoderParams(ctypes.Structure):
    """dgpu_decoder_params (include/dirac_gpu.h)."""

    _fields_ = [("cformat", ctypes.c_int), ("width", ctypes.c_int), ("height", ctypes.c_int),
                ("luma_depth", ctypes.c_int), ("chroma_depth", ctypes.c_int), ("wlt_depth", ctypes.c_int),
                ("spatial_partition", ctypes.c_int), ("bp", BlockParams)]


class DecodeInput(ctypes.Structure):
    """dgpu_decode_input (include/dirac_gpu.h)."""

    _fields_ = [("pnum", ctypes.c_int), ("intra", ctypes.c_int), ("num_refs", ctypes.c_int), ("ref1", ctypes.c_int),
                ("ref2", ctypes.c_int), ("filter", ctypes.c_int), ("zero_residual", ctypes.c_int),
                ("band_qidx", ctypes.c_void_p), ("band_skip", ctypes.c_void_p), ("on_host", ctypes.c_int),
                ("qindex", ctypes.c_void_p * 3), ("cb_skip", ctypes.c_void_p), ("mv1", ctypes.c_void_p),
                ("mv2", ctypes.c_void_p), ("mode", ctypes.c_void_p), ("dc", ctypes.c_void_p),
                ("split", ctypes.c_void_p), ("index_bits", ctypes.c_int)]


def block_params(width, height, precision, xblen, yblen, xbsep, ybsep):
    """Block parameters with the superblock counts of SequenceCompressor::SetMotionParameters
    (seq_compress.cpp:121-132)."""
    return BlockParams(precision=precision, xblen=xblen, yblen=yblen, xbsep=xbsep, ybsep=ybsep,
                       xnum_sb=(width + 4 * xbsep - 1) // (4 * xbsep),
                       ynum_sb=(height + 4 * ybsep - 1) // (4 * ybsep))


def decoder_params(cfg):
    """DecoderParams from encoder parameters (the dict SequenceEncoder takes)."""
    bp = block_params(cfg["width"], cfg["height"], cfg["mv_precision"], cfg["xblen"], cfg["yblen"], cfg["xbsep"],
                      cfg["ybsep"])
    return DecoderParams(cformat=cfg["cformat"], width=cfg["width"], height=cfg["height"],
                         luma_depth=cfg["luma_depth"], chroma_depth=cfg["chroma_depth"], wlt_depth=cfg["wlt_depth"],
                         spatial_partition=1, bp=bp)


def device_bytes(params, max_pictures=16):
    n = _lib.load().dgpu_decoder_device_bytes(ctypes.byref(params), max_pictures)
    if n == 0:
        raise ValueError("invalid decoder parameters")
    return n


def _host_ptr(a, dtype, keep):
    a = np.ascontiguousarray(a, dtype=dtype)
    keep.append(a)
    return a.ctypes.data


def _dev_ptr(t, dtype, keep):
    t = t.contiguous()
    if t.dtype != dtype:
        raise TypeError(f"expected {dtype}, got {t.dtype}")
    keep.append(t)
    return t.data_ptr()


class SequenceDecoder:
    """One decoded sequence on one CUDA stream; max_pictures device picture slots (the
    picture buffer: release() frees one)."""

    def __init__(self, params, max_pictures=16, stream=None):
        self.lib = _lib.load()
        self.params = params
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        self.handle = ctypes.c_void_p()
        _lib.check(self.lib.dgpu_decoder_create(ctypes.byref(self.params), max_pictures, self.stream.cuda_stream,
                                                ctypes.byref(self.handle)), "dgpu_decoder_create")
        p = self.params
        self.depth8 = p.luma_depth <= 8 and p.chroma_depth <= 8
        self._keep = []

    def close(self):
        if self.handle:
            self.lib.dgpu_decoder_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def prepare(self, pnum, intra, refs, filt, qindex, bands, cb_skip, motion=None, zero_residual=False):
        """The dgpu_decode_input of one picture (and the arrays it points to, which must stay
        alive while it is used): see decode."""
        keep = []
        on_host = not isinstance(qindex[0], torch.Tensor)
        b = [np.asarray(x, np.int32).reshape(-1, np.asarray(x).size // (3 * self.params.wlt_depth + 1))
             for x in bands]
        bq = np.ascontiguousarray(np.concatenate([x[:, 0] for x in b]), np.int32)
        bs = np.ascontiguousarray(np.concatenate([x[:, 1] for x in b]), np.int32)
        keep += [bq, bs]
        # int16 index arrays (numpy or torch) go as they are: half the bytes copied
        q0 = qindex[0]
        idx16 = q0.dtype == torch.int16 if isinstance(q0, torch.Tensor) else np.asarray(q0).dtype == np.int16
        I = DecodeInput(pnum=pnum, intra=int(bool(intra)), num_refs=len(refs), ref1=refs[0] if refs else -1,
                        ref2=refs[1] if len(refs) > 1 else -1, filter=filt, zero_residual=int(bool(zero_residual)),
                        band_qidx=bq.ctypes.data, band_skip=bs.ctypes.data, on_host=int(on_host),
                        index_bits=16 if idx16 else 32)
        if on_host:
            for c in range(3):
                I.qindex[c] = _host_ptr(qindex[c], np.int16 if idx16 else np.int32, keep)
            flags = cb_skip if isinstance(cb_skip, np.ndarray) else \
                np.concatenate([np.asarray(x, np.uint8).ravel() for x in cb_skip])
            I.cb_skip = _host_ptr(flags, np.uint8, keep)
        else:
            for c in range(3):
                I.qindex[c] = _dev_ptr(qindex[c], torch.int16 if idx16 else torch.int32, keep)
            flags = cb_skip if isinstance(cb_skip, torch.Tensor) else torch.cat([x.reshape(-1) for x in cb_skip])
            I.cb_skip = _dev_ptr(flags, torch.uint8, keep)
        if not intra:
            mv = motion["mv"]
            ptr = _host_ptr if on_host else _dev_ptr
            t16, t8 = (np.int16, np.uint8) if on_host else (torch.int16, torch.uint8)
            I.mv1 = ptr(mv[0], t16, keep)
            I.mv2 = ptr(mv[1], t16, keep) if len(refs) > 1 else None
            I.mode = ptr(motion["mode"], t8, keep)
            I.dc = ptr(motion["dc"], t16, keep)
            I.split = ptr(motion["split"], t8, keep)
        return I, keep

    def decode_prepared(self, prepared):
        _lib.check(self.lib.dgpu_decoder_decode(self.handle, ctypes.byref(prepared[0])), "dgpu_decoder_decode")

    def decode(self, pnum, intra, refs, filt, qindex, bands, cb_skip, motion=None, zero_residual=False):
        """Decodes one picture.

        qindex: three int32 [ch][cw] index arrays (numpy: host inputs; CUDA tensors: device
        inputs), or int16 ones when every index fits (index_bits 16); bands: three [3*depth+1][>=2] arrays of (quantiser index, skip, ...) per band
        (the DGPU_ENC_BANDS layout); cb_skip: three uint8 code-block flag arrays, or one with
        the three concatenated (host or device like qindex); motion (inter): {"mv": [mv1, mv2?]
        int16 [blocks][2], "mode", "dc" int16 [3][blocks], "split"}, host or device like
        qindex."""
        prepared = self.prepare(pnum, intra, refs, filt, qindex, bands, cb_skip, motion, zero_residual)
        self.decode_prepared(prepared)
        # inputs are read by work queued on the stream: keep them alive until a read
        # synchronises it
        self._keep.append(prepared)

    def release(self, pnum):
        _lib.check(self.lib.dgpu_decoder_release(self.handle, pnum), "dgpu_decoder_release")

    def read(self, pnum, what, comp=0):
        """RECON (int16 codec samples), COEFF (int32) or OUTPUT (unsigned samples) as numpy."""
        n = self.lib.dgpu_decoder_item_bytes(self.handle, pnum, what, comp)
        if n == 0:
            return None
        dt = {RECON: np.int16, COEFF: np.int32}.get(what, np.uint8 if self.depth8 else np.uint16)
        out = np.empty(n // np.dtype(dt).itemsize, dt)
        _lib.check(self.lib.dgpu_decoder_read(self.handle, pnum, what, comp, out.ctypes.data, n, 1),
                   "dgpu_decoder_read")
        self._keep = []
        return out

    def read_into(self, pnum, what, comp, dst):
        """Copies one result into a CUDA tensor or pinned host tensor of the right size."""
        n = self.lib.dgpu_decoder_item_bytes(self.handle, pnum, what, comp)
        if n == 0 or dst.numel() * dst.element_size() != n:
            raise ValueError("destination size does not match the item")
        _lib.check(self.lib.dgpu_decoder_read(self.handle, pnum, what, comp, dst.data_ptr(), n,
                                              int(not dst.is_cuda)), "dgpu_decoder_read")


def dequantise(intra, depth, qindex, bands, ncb, cb_skip, out=None, stream=None):
    """dgpu_dequantise_batch over CUDA tensors: qindex (list of int32 [ch][cw], or int16 for
    dgpu_dequantise_batch16), bands (per component [3*depth+1][>=2] quantiser index, skip), ncb
    (per component the [nb][2] code block counts), cb_skip (per component uint8 flags, CUDA).
    Returns the int32 coefficients."""
    lib = _lib.load()
    n = len(qindex)
    intra = list(intra) if hasattr(intra, "__len__") else [intra] * n
    depth = list(depth) if hasattr(depth, "__len__") else [depth] * n
    q = [t.contiguous() for t in qindex]
    idx16 = q[0].dtype == torch.int16
    if any(t.dtype != q[0].dtype for t in q) or q[0].dtype not in (torch.int16, torch.int32):
        raise TypeError("qindex: int32 or int16 tensors of one type")
    out = out if out is not None else [torch.empty(t.shape, dtype=torch.int32, device=t.device) for t in q]
    b = [np.asarray(x, np.int32).reshape(3 * d + 1, -1) for x, d in zip(bands, depth)]
    bq = np.ascontiguousarray(np.concatenate([x[:, 0] for x in b]), np.int32)
    bs = np.ascontiguousarray(np.concatenate([x[:, 1] for x in b]), np.int32)
    nc = np.ascontiguousarray(np.concatenate([np.asarray(x, np.int32).ravel() for x in ncb]), np.int32)
    cbs = torch.cat([x.reshape(-1) for x in cb_skip]).contiguous()
    st = stream if stream is not None else torch.cuda.current_stream()
    fn = lib.dgpu_dequantise_batch16 if idx16 else lib.dgpu_dequantise_batch
    rc = fn(
        n, _lib.int_array(intra), _lib.int_array(depth), _lib.ptr_array([t.data_ptr() for t in q]),
        _lib.ptr_array([t.data_ptr() for t in out]), _lib.int_array([t.shape[1] for t in q]),
        _lib.int_array([t.shape[0] for t in q]), nc.ctypes.data_as(_lib.P_int), bq.ctypes.data_as(_lib.P_int),
        bs.ctypes.data_as(_lib.P_int), cbs.data_ptr(), st.cuda_stream)
    _lib.check(rc, "dgpu_dequantise_batch16" if idx16 else "dgpu_dequantise_batch")
    return out
