"""Host-side mirror of the reference's sequence coding loop over the library's device encoder.

``SequenceEncoder`` wraps the dgpu_encoder_* entry points: pictures are loaded in display
order (dirac_encoder_load, libdirac_encoder/dirac_encoder.cpp:1067-1087), coded one at a time
in coding order (SequenceCompressor::CompressNextPicture, seq_compress.cpp:194-499) and their
results read back per picture.  The arithmetic coder is not part of this path: the caller
supplies entropy-correction factors per picture, or the encoder keeps the initial ones.
"""
import ctypes

import numpy as np
import torch

from . import _lib

RECON, COEFF, QINDEX, MV, MODE, DC, SPLIT, BANDS, CBSKIP, OUTPUT = range(10)
STAGES = ["load", "motion_estimation", "mc_subtract", "dwt_forward", "quantisation", "dwt_inverse",
          "mc_add_clip", "upconvert"]


class EncoderParams(ctypes.Structure):
    """dgpu_encoder_params (include/dirac_gpu.h)."""

    _fields_ = [("cformat", ctypes.c_int), ("width", ctypes.c_int), ("height", ctypes.c_int),
                ("luma_depth", ctypes.c_int), ("chroma_depth", ctypes.c_int), ("qf", ctypes.c_float),
                ("l1_sep", ctypes.c_int), ("num_l1", ctypes.c_int), ("cpd", ctypes.c_float),
                ("xblen", ctypes.c_int), ("yblen", ctypes.c_int), ("xbsep", ctypes.c_int), ("ybsep", ctypes.c_int),
                ("mv_precision", ctypes.c_int), ("intra_filter", ctypes.c_int), ("inter_filter", ctypes.c_int),
                ("wlt_depth", ctypes.c_int), ("field_coding", ctypes.c_int), ("top_field_first", ctypes.c_int)]


class PictureInfo(ctypes.Structure):
    """dgpu_picture_info (include/dirac_gpu.h)."""

    _fields_ = [("pnum", ctypes.c_int), ("coded_num", ctypes.c_int), ("intra", ctypes.c_int),
                ("is_ref", ctypes.c_int), ("cut", ctypes.c_int), ("num_refs", ctypes.c_int), ("ref1", ctypes.c_int),
                ("ref2", ctypes.c_int), ("is_b", ctypes.c_int), ("filter", ctypes.c_int),
                ("intra_ratio", ctypes.c_double), ("cpd_scale", ctypes.c_double), ("lambda_", ctypes.c_float * 3)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "lambda_"}
        d["lambda"] = list(self.lambda_)
        return d


_DTYPES = {RECON: np.int16, COEFF: np.int32, QINDEX: np.int32, MV: np.int16, MODE: np.uint8, DC: np.int16,
           SPLIT: np.uint8, BANDS: np.int32, CBSKIP: np.uint8}


def device_bytes(params, max_pictures=32):
    """Device memory a SequenceEncoder with these parameters allocates (no GPU needed)."""
    p = EncoderParams(**params)
    n = _lib.load().dgpu_encoder_device_bytes(ctypes.byref(p), max_pictures)
    if n == 0:
        raise ValueError("invalid encoder parameters")
    return n


class SequenceEncoder:
    """One coded sequence on one CUDA stream.

    params: dict with the EncoderParams fields (cformat, width, height, luma_depth,
    chroma_depth, qf, l1_sep, num_l1, cpd, xblen, yblen, xbsep, ybsep, mv_precision,
    intra_filter, inter_filter, wlt_depth).  max_pictures: device picture slots."""

    def __init__(self, params, max_pictures=32, stream=None):
        self.lib = _lib.load()
        self.params = EncoderParams(**params)
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        self.handle = ctypes.c_void_p()
        _lib.check(self.lib.dgpu_encoder_create(ctypes.byref(self.params), max_pictures, self.stream.cuda_stream,
                                                ctypes.byref(self.handle)), "dgpu_encoder_create")
        p = self.params
        self.depth8 = p.luma_depth <= 8 and p.chroma_depth <= 8
        xs = 0 if p.cformat == 0 else 1
        ys = 1 if p.cformat == 2 else 0
        h = p.height // 2 if p.field_coding else p.height  # a picture is a field when field coding
        self.shapes = [(h, p.width), (h >> ys, p.width >> xs), (h >> ys, p.width >> xs)]

    def close(self):
        if self.handle:
            self.lib.dgpu_encoder_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, planes):
        """planes: three unsigned sample planes (numpy arrays in host memory, or CUDA tensors)."""
        on_host = not isinstance(planes[0], torch.Tensor)
        if on_host:
            dt = np.uint8 if self.depth8 else np.uint16
            arrs = [np.ascontiguousarray(a, dtype=dt) for a in planes]
            ptrs = [a.ctypes.data for a in arrs]
        else:
            ptrs = [t.data_ptr() for t in planes]
        _lib.check(self.lib.dgpu_encoder_load(self.handle, _lib.ptr_array(ptrs), int(on_host)), "dgpu_encoder_load")

    def reset(self):
        """Start a new sequence, keeping the device memory."""
        _lib.check(self.lib.dgpu_encoder_reset(self.handle), "dgpu_encoder_reset")

    def profile(self, enable):
        """Turn stage timing on/off; returns {stage: (ms, calls)} accumulated so far."""
        ms = (ctypes.c_double * len(STAGES))()
        calls = (ctypes.c_int * len(STAGES))()
        _lib.check(self.lib.dgpu_encoder_profile(self.handle, int(enable), ms, calls), "dgpu_encoder_profile")
        return {n: (ms[k], calls[k]) for k, n in enumerate(STAGES)}

    def end_sequence(self):
        _lib.check(self.lib.dgpu_encoder_end_sequence(self.handle), "dgpu_encoder_end_sequence")

    def code_next(self, ecf=None, ecf_state=None):
        """Codes the next picture in coding order; returns its info dict, or None.  ecf: the
        picture's [3][3*depth+1] entropy-correction factors; ecf_state: instead, a whole
        EntropyCorrector state (entropy.EntropyCorrector.state), from which the encoder picks
        the picture's factors once its kind is final."""
        info = PictureInfo()
        if ecf_state is not None:
            st = np.ascontiguousarray(ecf_state, dtype=np.float32)
            rc = self.lib.dgpu_encoder_code_next_adaptive(self.handle, st.ctypes.data, ctypes.byref(info))
            if rc < 0:
                _lib.check(rc, "dgpu_encoder_code_next_adaptive")
            return info.as_dict() if rc == 1 else None
        e = None
        if ecf is not None:
            e = np.ascontiguousarray(ecf, dtype=np.float32)
        rc = self.lib.dgpu_encoder_code_next(self.handle, e.ctypes.data if e is not None else None, ctypes.byref(info))
        if rc < 0:
            _lib.check(rc, "dgpu_encoder_code_next")
        return info.as_dict() if rc == 1 else None

    def prepare_next(self):
        """First half of code_next (no entropy factors needed): returns the prepared picture's
        info (kind final), or None when more input is needed."""
        info = PictureInfo()
        rc = self.lib.dgpu_encoder_prepare_next(self.handle, ctypes.byref(info))
        if rc < 0:
            _lib.check(rc, "dgpu_encoder_prepare_next")
        return info.as_dict() if rc == 1 else None

    def finish_next(self, ecf=None, ecf_state=None):
        """Second half: quantiser choice with ecf (or the kind's factors from ecf_state),
        quantisation, reconstruction.  Returns the picture's final info."""
        info = PictureInfo()
        e = np.ascontiguousarray(ecf, dtype=np.float32) if ecf is not None else None
        st = np.ascontiguousarray(ecf_state, dtype=np.float32) if ecf_state is not None else None
        rc = self.lib.dgpu_encoder_finish_next(self.handle, e.ctypes.data if e is not None else None,
                                               st.ctypes.data if st is not None else None, ctypes.byref(info))
        _lib.check(rc if rc < 0 else 0, "dgpu_encoder_finish_next")
        return info.as_dict()

    def read(self, pnum, what, comp=0):
        """One result of a coded picture as a numpy array."""
        n = self.lib.dgpu_encoder_item_bytes(self.handle, pnum, what, comp)
        if n == 0:
            return None
        if what == OUTPUT:
            dt = np.uint8 if self.depth8 else np.uint16
        else:
            dt = _DTYPES[what]
        out = np.empty(n // np.dtype(dt).itemsize, dt)
        _lib.check(self.lib.dgpu_encoder_read(self.handle, pnum, what, comp, out.ctypes.data, n, 1), "dgpu_encoder_read")
        return out

    def encode(self, frames):
        """Loads every frame, ends the sequence and codes all pictures; returns the infos in
        coding order."""
        for f in frames:
            self.load(f)
        self.end_sequence()
        infos = []
        while True:
            i = self.code_next()
            if i is None:
                return infos
            infos.append(i)


class EncoderGroup:
    """Several SequenceEncoders (same picture size, chroma format, luma depth and block
    parameters) whose motion estimation runs in one batched launch: after each member has
    loaded its pictures, estimate() estimates every member's inter pictures whose references
    are known; the members' code_next calls then reuse those estimates."""

    def __init__(self, encoders):
        self.lib = _lib.load()
        self.members = list(encoders)
        self.handle = ctypes.c_void_p()
        hs = _lib.ptr_array([e.handle.value for e in self.members])
        _lib.check(self.lib.dgpu_encoder_group_create(hs, len(self.members), ctypes.byref(self.handle)),
                   "dgpu_encoder_group_create")

    def estimate(self):
        """Runs the batched estimation; returns the number of picture estimates made."""
        n = ctypes.c_int(0)
        _lib.check(self.lib.dgpu_encoder_group_estimate(self.handle, ctypes.byref(n)), "dgpu_encoder_group_estimate")
        return n.value

    def close(self):
        if self.handle:
            self.lib.dgpu_encoder_group_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
