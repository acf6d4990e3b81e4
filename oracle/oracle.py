"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU checkers built by oracle/Makefile.

``Oracle`` wraps liboracle.so, this project's plain-C restatement of the Dirac hot path
(oracle/dirac_oracle.c).  ``Reference`` wraps oracle/_ref/libdirac_ref.so, the reference
codec's own C++ compiled from its sources plus the stage driver oracle/ref_driver.cpp; it
exists only where the reference sources were available at build time.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use this module.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libdirac_ref.so")


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def padded(w, h, depth):
    mul = 1 << depth
    return (w + mul - 1) // mul * mul, (h + mul - 1) // mul * mul


class Oracle:
    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle oracle`")
        self.lib = ctypes.CDLL(path)

    def dwt_min_len(self, filt):
        return self.lib.orc_dwt_min_len(filt)

    def dwt_forward(self, filt, depth, pic, cw=None, ch=None):
        pic = np.ascontiguousarray(pic, dtype=np.int16)
        h, w = pic.shape
        if cw is None:
            cw, ch = padded(w, h, depth)
        coeff = np.zeros((ch, cw), np.int32)
        rc = self.lib.orc_dwt_forward(filt, depth, _p(pic), w, h, w, _p(coeff), cw, ch, cw)
        if rc:
            raise ValueError(f"orc_dwt_forward rc={rc}")
        return coeff

    def dwt_backward(self, filt, depth, coeff, w, h):
        c = np.array(coeff, dtype=np.int32, copy=True, order="C")
        ch, cw = c.shape
        pic = np.zeros((h, w), np.int16)
        rc = self.lib.orc_dwt_backward(filt, depth, _p(c), cw, ch, cw, _p(pic), w, h, w)
        if rc:
            raise ValueError(f"orc_dwt_backward rc={rc}")
        return pic

    def upconvert(self, pic, bit_depth):
        pic = np.ascontiguousarray(pic, dtype=np.int16)
        h, w = pic.shape
        up = np.zeros((2 * h, 2 * w), np.int16)
        rc = self.lib.orc_upconvert(_p(pic), w, h, w, bit_depth, _p(up), 2 * w)
        if rc:
            raise ValueError(f"orc_upconvert rc={rc}")
        return up

    def downconvert(self, pic):
        pic = np.ascontiguousarray(pic, dtype=np.int16)
        h, w = pic.shape
        out = np.zeros((h // 2, w // 2), np.int16)
        rc = self.lib.orc_downconvert(_p(pic), w, h, w, _p(out), w // 2)
        if rc:
            raise ValueError(f"orc_downconvert rc={rc}")
        return out


class Reference:
    """The reference codec itself (plain-C build), driven stage by stage."""

    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle` where the reference sources exist")
        self.lib = ctypes.CDLL(path)

    @staticmethod
    def available(path=REF_SO):
        return os.path.exists(path)

    def dwt_forward(self, filt, depth, pic, cw=None, ch=None):
        pic = np.ascontiguousarray(pic, dtype=np.int16)
        h, w = pic.shape
        if cw is None:
            cw, ch = padded(w, h, depth)
        coeff = np.zeros((ch, cw), np.int32)
        if self.lib.ref_dwt_forward(filt, depth, _p(pic), w, h, _p(coeff), cw, ch):
            raise ValueError("ref_dwt_forward failed")
        return coeff

    def dwt_backward(self, filt, depth, coeff, w, h):
        c = np.array(coeff, dtype=np.int32, copy=True, order="C")
        ch, cw = c.shape
        pic = np.zeros((h, w), np.int16)
        if self.lib.ref_dwt_backward(filt, depth, _p(c), cw, ch, _p(pic), w, h):
            raise ValueError("ref_dwt_backward failed")
        return pic

    def upconvert(self, pic, bit_depth):
        pic = np.ascontiguousarray(pic, dtype=np.int16)
        h, w = pic.shape
        up = np.zeros((2 * h, 2 * w), np.int16)
        if self.lib.ref_upconvert(_p(pic), w, h, bit_depth, _p(up)):
            raise ValueError("ref_upconvert failed")
        return up

    def downconvert(self, pic):
        pic = np.ascontiguousarray(pic, dtype=np.int16)
        h, w = pic.shape
        out = np.zeros((h // 2, w // 2), np.int16)
        if self.lib.ref_downconvert(_p(pic), w, h, _p(out)):
            raise ValueError("ref_downconvert failed")
        return out
