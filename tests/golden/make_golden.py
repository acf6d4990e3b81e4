"""Generate the golden fixtures in this directory by running the reference codec itself.

Needs oracle/_ref/libdirac_ref.so (the reference's own C++, plain-C build, compiled from
its sources by `make -C oracle`).  Inputs are seeded, so re-running reproduces the files.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
from oracle import Reference  # noqa: E402


def dwt_cases(ref):
    rng = np.random.default_rng(20261203)
    out = {}
    # (w, h, depth): odd padding on both axes; level sides stay >= 6
    shapes = [(70, 38, 3), (45, 52, 2), (64, 48, 4)]
    for filt in range(7):
        for k, (w, h, depth) in enumerate(shapes):
            mul = 1 << depth
            cw, ch = (w + mul - 1) // mul * mul, (h + mul - 1) // mul * mul
            pic = rng.integers(-128, 128, size=(h, w)).astype(np.int16)
            coeff = ref.dwt_forward(filt, depth, pic, cw, ch)
            noisy = (coeff + rng.integers(-9, 10, size=coeff.shape)).astype(np.int32)
            back = ref.dwt_backward(filt, depth, noisy, w, h)
            key = f"f{filt}_c{k}"
            out[key + "_pic"] = pic
            out[key + "_coeff"] = coeff
            out[key + "_noisy"] = noisy
            out[key + "_back"] = back
            out[key + "_meta"] = np.array([filt, depth, w, h, cw, ch], np.int32)
    return out


def conv_cases(ref):
    rng = np.random.default_rng(7)
    out = {}
    for k, (w, h, bd) in enumerate([(40, 24, 8), (33, 17, 10), (8, 8, 8)]):
        pic = rng.integers(-(1 << (bd - 1)), 1 << (bd - 1), size=(h, w)).astype(np.int16)
        out[f"up{k}_pic"] = pic
        out[f"up{k}_out"] = ref.upconvert(pic, bd)
        out[f"up{k}_meta"] = np.array([w, h, bd], np.int32)
    for k, (w, h) in enumerate([(64, 50), (49, 31), (24, 24)]):
        pic = rng.integers(-128, 128, size=(h, w)).astype(np.int16)
        out[f"down{k}_pic"] = pic
        out[f"down{k}_out"] = ref.downconvert(pic)
    return out


def main():
    ref = Reference()
    np.savez_compressed(os.path.join(HERE, "dwt.npz"), **dwt_cases(ref))
    np.savez_compressed(os.path.join(HERE, "convert.npz"), **conv_cases(ref))
    print("wrote dwt.npz, convert.npz")


if __name__ == "__main__":
    main()
