"""Host-side mirrors of the reference's up/down-conversion and motion-compensation calls
over device tensors (int16 CUDA tensors; see include/dirac_gpu.h for the contracts).

References: UpConverter::DoUpConverter (libdirac_common/upconvert.cpp:55-200),
DownConverter::DoDownConvert (libdirac_motionest/downconvert.cpp:51-204),
MotionCompensator::CompensatePicture (libdirac_common/mot_comp.cpp:63-192).
"""
import ctypes

import torch

from . import _lib
from ._lib import BlockParams

ADD, SUBTRACT = 0, 1
INTRA, REF1_ONLY, REF2_ONLY, REF1AND2 = 0, 1, 2, 3
FORMAT444, FORMAT422, FORMAT420 = 0, 1, 2


def chroma_shift(cformat):
    return {0: (0, 0), 1: (1, 0), 2: (1, 1)}[cformat]


def _sp(stream):
    return (stream if stream is not None else torch.cuda.current_stream()).cuda_stream


def _i16(t, name):
    if not t.is_cuda or t.dtype != torch.int16 or t.dim() != 2 or t.stride(1) != 1:
        raise ValueError(f"{name} must be a 2-D int16 CUDA tensor with unit column stride")


def upconvert(pic, bit_depth, out=None, stream=None):
    """Half-pel upconversion of one component: returns a (2h, 2w) int16 tensor."""
    _i16(pic, "pic")
    h, w = pic.shape
    if out is None:
        out = torch.empty((2 * h, 2 * w), dtype=torch.int16, device=pic.device)
    rc = _lib.load().dgpu_upconvert(pic.data_ptr(), w, h, pic.stride(0), bit_depth, out.data_ptr(),
                                    out.stride(0), _sp(stream))
    _lib.check(rc, "dgpu_upconvert")
    return out


def upconvert_batch(pics, bit_depths, outs, stream=None):
    n = len(pics)
    rc = _lib.load().dgpu_upconvert_batch(
        n, _lib.ptr_array([p.data_ptr() for p in pics]), _lib.int_array([p.shape[1] for p in pics]),
        _lib.int_array([p.shape[0] for p in pics]), _lib.int_array([p.stride(0) for p in pics]),
        _lib.int_array(list(bit_depths)), _lib.ptr_array([o.data_ptr() for o in outs]),
        _lib.int_array([o.stride(0) for o in outs]), _sp(stream))
    _lib.check(rc, "dgpu_upconvert_batch")


def downconvert(pic, out=None, stream=None):
    """2x decimation: returns an (h//2, w//2) int16 tensor."""
    _i16(pic, "pic")
    h, w = pic.shape
    if out is None:
        out = torch.empty((h // 2, w // 2), dtype=torch.int16, device=pic.device)
    rc = _lib.load().dgpu_downconvert(pic.data_ptr(), w, h, pic.stride(0), out.data_ptr(), out.stride(0),
                                      _sp(stream))
    _lib.check(rc, "dgpu_downconvert")
    return out


def downconvert_batch(pics, outs, stream=None):
    n = len(pics)
    rc = _lib.load().dgpu_downconvert_batch(
        n, _lib.ptr_array([p.data_ptr() for p in pics]), _lib.int_array([p.shape[1] for p in pics]),
        _lib.int_array([p.shape[0] for p in pics]), _lib.int_array([p.stride(0) for p in pics]),
        _lib.ptr_array([o.data_ptr() for o in outs]), _lib.int_array([o.stride(0) for o in outs]), _sp(stream))
    _lib.check(rc, "dgpu_downconvert_batch")


def clip(pic, bit_depth, stream=None):
    _i16(pic, "pic")
    h, w = pic.shape
    _lib.check(_lib.load().dgpu_clip(pic.data_ptr(), w, h, pic.stride(0), bit_depth, _sp(stream)), "dgpu_clip")


class MotionCompensator:
    """Mirror of MotionCompensator::CompensatePicture(ppp, direction, mv_data, pic, refs).

    bp: BlockParams.  Block data are CUDA tensors: mv1/mv2 int16 (ynb, xnb, 2), mode uint8
    (ynb, xnb), dc int16 (3, ynb, xnb), split uint8 (ynsb, xnsb)."""

    def __init__(self, bp, cformat=FORMAT420):
        self.lib = _lib.load()
        self.bp = bp
        self.cformat = cformat

    def CompensatePicture(self, direction, mv1, mv2, mode, dc, split, pic, ref1up, ref2up=None,
                          clip_depths=(0, 0), stream=None, weights=(1, 1, 1)):
        """weights: the picture's reference weights (ref1, ref2, precision bits)."""
        for t in pic:
            _i16(t, "pic")
        h, w = pic[0].shape
        ups2 = ref2up if ref2up is not None else ref1up
        rc = self.lib.dgpu_motion_compensate_weighted(
            direction, self.cformat, w, h, ctypes.byref(self.bp), mv1.data_ptr(),
            mv2.data_ptr() if mv2 is not None else None, mode.data_ptr(), dc.data_ptr(), split.data_ptr(),
            _lib.ptr_array([p.data_ptr() for p in pic]), _lib.int_array([p.stride(0) for p in pic]),
            _lib.ptr_array([u.data_ptr() for u in ref1up]), _lib.ptr_array([u.data_ptr() for u in ups2]),
            clip_depths[0], clip_depths[1], int(weights[0]), int(weights[1]), int(weights[2]), _sp(stream))
        _lib.check(rc, "dgpu_motion_compensate_weighted")


class MotionEstimator:
    """Mirror of PictureCompressor::PixelME / SubPixelME / ModeDecisionME for one picture.

    Estimate(pic, ref1, ref2=None, lambda_=..., stages=3) takes the original component planes
    as int16 CUDA tensors and returns a dict of CUDA tensors: mv (nref, ynb, xnb, 2) int16,
    cost (nref, ynb, xnb, 3) float32 (SAD, mvcost, total), and after stage 3 mode (ynb, xnb)
    uint8, dc (3, ynb, xnb) int16, split / sbcost (ynsb, xnsb)."""

    def __init__(self, bp, cformat=FORMAT420, luma_depth=8):
        self.lib = _lib.load()
        self.bp = bp
        self.cformat = cformat
        self.luma_depth = luma_depth

    def Estimate(self, pic, ref1, ref2=None, lambda_=10.0, stages=3, stream=None):
        for t in list(pic) + list(ref1) + (list(ref2) if ref2 is not None else []):
            _i16(t, "plane")
            if not t.is_contiguous():
                raise ValueError("motion estimation planes must be dense")
        nref = 2 if ref2 is not None else 1
        h, w = pic[0].shape
        bp = self.bp
        ynb, xnb = 4 * bp.ynum_sb, 4 * bp.xnum_sb
        dev = pic[0].device
        out = {
            "mv": torch.zeros((nref, ynb, xnb, 2), dtype=torch.int16, device=dev),
            "cost": torch.zeros((nref, ynb, xnb, 3), dtype=torch.float32, device=dev),
            "mode": torch.zeros((ynb, xnb), dtype=torch.uint8, device=dev),
            "dc": torch.zeros((3, ynb, xnb), dtype=torch.int16, device=dev),
            "split": torch.zeros((bp.ynum_sb, bp.xnum_sb), dtype=torch.uint8, device=dev),
            "sbcost": torch.zeros((bp.ynum_sb, bp.xnum_sb), dtype=torch.float32, device=dev),
        }
        r2 = ref2 if ref2 is not None else ref1
        rc = self.lib.dgpu_motion_estimate(
            self.cformat, w, h, ctypes.byref(bp), nref, _lib.ptr_array([p.data_ptr() for p in pic]),
            _lib.ptr_array([p.data_ptr() for p in ref1]), _lib.ptr_array([p.data_ptr() for p in r2]),
            self.luma_depth, ctypes.c_float(lambda_), stages, out["mv"].data_ptr(), out["cost"].data_ptr(),
            out["mode"].data_ptr(), out["dc"].data_ptr(), out["split"].data_ptr(), out["sbcost"].data_ptr(),
            None, 0, _sp(stream))
        _lib.check(rc, "dgpu_motion_estimate")
        return out

    def EstimateBatch(self, pics, tasks, stages=3, stream=None, outs=None):
        """Batched motion estimation.  pics: list of 3-plane pictures (dense int16 CUDA
        tensors); tasks: list of (pic index, ref1 index, ref2 index or -1, lambda).  Returns
        (or fills, when outs is given) one output dict per task, as Estimate does."""
        bp = self.bp
        h, w = pics[0][0].shape
        ynb, xnb = 4 * bp.ynum_sb, 4 * bp.xnum_sb
        dev = pics[0][0].device
        if outs is None:
            outs = [self.new_outputs(dev) for _ in tasks]
        planes = [p for pic in pics for p in pic]
        for t in planes:
            _i16(t, "plane")
        n = len(tasks)
        rc = self.lib.dgpu_motion_estimate_batch(
            self.cformat, w, h, ctypes.byref(bp), self.luma_depth, len(pics),
            _lib.ptr_array([p.data_ptr() for p in planes]), n,
            _lib.int_array([t[0] for t in tasks]), _lib.int_array([t[1] for t in tasks]),
            _lib.int_array([t[2] for t in tasks]),
            (ctypes.c_float * n)(*[t[3] for t in tasks]), stages,
            _lib.ptr_array([o["mv"].data_ptr() for o in outs]), _lib.ptr_array([o["cost"].data_ptr() for o in outs]),
            _lib.ptr_array([o["mode"].data_ptr() for o in outs]), _lib.ptr_array([o["dc"].data_ptr() for o in outs]),
            _lib.ptr_array([o["split"].data_ptr() for o in outs]),
            _lib.ptr_array([o["sbcost"].data_ptr() for o in outs]), None, 0, _sp(stream))
        _lib.check(rc, "dgpu_motion_estimate_batch")
        return outs

    def new_outputs(self, dev):
        bp = self.bp
        ynb, xnb = 4 * bp.ynum_sb, 4 * bp.xnum_sb
        return {
            "mv": torch.zeros((2, ynb, xnb, 2), dtype=torch.int16, device=dev),
            "cost": torch.zeros((2, ynb, xnb, 3), dtype=torch.float32, device=dev),
            "mode": torch.zeros((ynb, xnb), dtype=torch.uint8, device=dev),
            "dc": torch.zeros((3, ynb, xnb), dtype=torch.int16, device=dev),
            "split": torch.zeros((bp.ynum_sb, bp.xnum_sb), dtype=torch.uint8, device=dev),
            "sbcost": torch.zeros((bp.ynum_sb, bp.xnum_sb), dtype=torch.float32, device=dev),
        }
