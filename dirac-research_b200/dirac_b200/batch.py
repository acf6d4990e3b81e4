"""Heterogeneous picture batch (dgpu_batch_*): many pictures of different sizes, chroma
formats, bit depths, filters and depths coded together, each as PictureCompressor codes one
picture once its motion data is known (libdirac_encoder/picture_compress.cpp:92-180,
418-531): motion compensation SUBTRACT, forward transform, quantiser choice with quantisation
and reconstruction, inverse transform, motion compensation ADD with the clip (or the clip)."""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import BlockParams
from .encoder import _DTYPES, BANDS, CBSKIP, COEFF, QINDEX, RECON


class BatchPicture(ctypes.Structure):
    """dgpu_batch_picture (include/dirac_gpu.h)."""

    _fields_ = [("cformat", ctypes.c_int), ("width", ctypes.c_int), ("height", ctypes.c_int),
                ("luma_depth", ctypes.c_int), ("chroma_depth", ctypes.c_int), ("filter", ctypes.c_int),
                ("wlt_depth", ctypes.c_int), ("intra", ctypes.c_int), ("is_b", ctypes.c_int),
                ("qf", ctypes.c_float), ("cpd", ctypes.c_float), ("intra_ratio", ctypes.c_double),
                ("bp", BlockParams)]


class BatchMotion(ctypes.Structure):
    """dgpu_batch_motion (include/dirac_gpu.h)."""

    _fields_ = [("ref1", ctypes.c_void_p * 3), ("ref2", ctypes.c_void_p * 3), ("mv1", ctypes.c_void_p),
                ("mv2", ctypes.c_void_p), ("mode", ctypes.c_void_p), ("dc", ctypes.c_void_p),
                ("split", ctypes.c_void_p)]


def _picture(d):
    p = BatchPicture()
    for k in ("cformat", "width", "height", "luma_depth", "chroma_depth", "filter", "wlt_depth", "intra", "is_b"):
        setattr(p, k, int(d.get(k, 0)))
    p.qf = float(d.get("qf", 7.0))
    p.cpd = float(d.get("cpd", 32.0))
    p.intra_ratio = float(d.get("intra_ratio", 0.0))
    if "bp" in d:
        p.bp = d["bp"]
    return p


def _motion(m):
    """m: dict of CUDA tensors: ref1 / ref2 (three int16 planes each, ref2 optional), mv1, mv2
    (optional), mode, dc, split; or None for an intra picture."""
    r = BatchMotion()
    if m is None:
        return r
    for c in range(3):
        r.ref1[c] = m["ref1"][c].data_ptr()
        if m.get("ref2") is not None:
            r.ref2[c] = m["ref2"][c].data_ptr()
    r.mv1 = m["mv1"].data_ptr()
    r.mv2 = m["mv2"].data_ptr() if m.get("mv2") is not None else None
    r.mode = m["mode"].data_ptr()
    r.dc = m["dc"].data_ptr()
    r.split = m["split"].data_ptr()
    return r


def device_bytes(pictures, motion=None):
    lib = _lib.load()
    n = len(pictures)
    pa = (BatchPicture * n)(*[_picture(d) for d in pictures])
    ma = (BatchMotion * n)(*[_motion(m) for m in motion]) if motion is not None else None
    return lib.dgpu_batch_device_bytes(n, pa, ma)


class PictureBatch:
    """pictures: list of dicts with the dgpu_batch_picture fields (bp: a BlockParams);
    motion: list of motion dicts (see _motion) or None per picture.  The motion tensors must
    stay alive while the batch does (the library keeps their device pointers)."""

    def __init__(self, pictures, motion=None, stream=None):
        self.lib = _lib.load()
        n = len(pictures)
        self.n = n
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        self._keep = motion
        pa = (BatchPicture * n)(*[_picture(d) for d in pictures])
        ma = (BatchMotion * n)(*[_motion(m) for m in (motion or [None] * n)])
        self.handle = ctypes.c_void_p()
        _lib.check(self.lib.dgpu_batch_create(n, pa, ma, self.stream.cuda_stream, ctypes.byref(self.handle)),
                   "dgpu_batch_create")
        self.pictures = pictures

    def planes(self, k):
        """Device pointers of picture k's three planes."""
        ptrs = (ctypes.c_void_p * 3)()
        _lib.check(self.lib.dgpu_batch_planes(self.handle, k, ptrs), "dgpu_batch_planes")
        return [ptrs[c] for c in range(3)]

    def load(self, k, planes):
        """Picture k's three planes: int16 codec samples as numpy arrays (host) or CUDA tensors."""
        on_host = not isinstance(planes[0], torch.Tensor)
        if on_host:
            arrs = [np.ascontiguousarray(a, dtype=np.int16) for a in planes]
            ptrs = [a.ctypes.data for a in arrs]
        else:
            ptrs = [t.data_ptr() for t in planes]
        _lib.check(self.lib.dgpu_batch_load(self.handle, k, _lib.ptr_array(ptrs), int(on_host)), "dgpu_batch_load")
        if on_host:
            torch.cuda.synchronize()  # pageable source arrays: complete the copies before they go

    def run(self):
        _lib.check(self.lib.dgpu_batch_run(self.handle), "dgpu_batch_run")

    def stage_times(self):
        """One run timed by stage: (pre-quantisation device work, quantisation, post) in ms."""
        ms = (ctypes.c_float * 3)()
        _lib.check(self.lib.dgpu_batch_stage_times(self.handle, ms), "dgpu_batch_stage_times")
        return list(ms)

    def read(self, k, what, comp=0):
        n = self.lib.dgpu_batch_item_bytes(self.handle, k, what, comp)
        if n == 0:
            return None
        dt = _DTYPES[what]
        out = np.empty(n // np.dtype(dt).itemsize, dt)
        _lib.check(self.lib.dgpu_batch_read(self.handle, k, what, comp, out.ctypes.data, n, 1), "dgpu_batch_read")
        return out

    def close(self):
        if self.handle:
            self.lib.dgpu_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["BatchPicture", "BatchMotion", "PictureBatch", "device_bytes", "RECON", "COEFF", "QINDEX", "BANDS",
           "CBSKIP"]
