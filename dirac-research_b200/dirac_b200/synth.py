"""Seeded synthetic video, the stand-in input for every workload (no public dataset).

Per plane: a smooth background (DC plus three random 2-D sinusoids with periods drawn from
[16, 128] px, each of amplitude 40/3 so that their sum stays within +-40), N rectangles
(sides drawn from [32, 96] px) textured with uniform noise over the full sample range and
moving at a constant velocity whose components are multiples of 1/4 px in [-vmax, vmax],
rendered at sub-pixel positions by bilinear resampling of the texture (positions wrap
around the frame so that content stays in view), then additive Gaussian noise of
sigma 2 (in 8-bit units) and a clip to [0, 2^bit_depth - 1].  Chroma planes use the same
generator at chroma resolution (DC at mid-range) with the rectangles' geometry scaled to
the chroma grid and their own textures.  Higher bit depths scale amplitudes by
2^(bit_depth-8).

Codec samples are signed: value - 2^(bit_depth-1), as the reference's picture reader
stores them (libdirac_common/pic_io.cpp:388-399 for 8-bit).
"""
import numpy as np

CHROMA = {"420": (2, 2), "422": (2, 1), "444": (1, 1)}


def _plane(rng, w, h, frames, rects, bit_depth, sx, sy):
    scale = float(1 << (bit_depth - 8))
    maxv = (1 << bit_depth) - 1
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)
    bg = np.full((h, w), 128.0 * scale)
    for _ in range(3):
        period = rng.uniform(16, 128)
        theta = rng.uniform(0, np.pi)
        phase = rng.uniform(0, 2 * np.pi)
        bg += (40.0 / 3.0) * scale * np.sin(2 * np.pi * (x * np.cos(theta) + y * np.sin(theta)) / period + phase)
    textures = [rng.integers(0, maxv + 1, size=(max(2, r[1] // sy), max(2, r[0] // sx))).astype(np.float64)
                for r in rects]
    out = []
    for t in range(frames):
        f = bg.copy()
        for (rw, rh, px, py, vx, vy), tex in zip(rects, textures):
            th, tw = tex.shape
            # top-left corner in this plane's grid, wrapping so the rectangle stays in view
            cx = ((px + vx * t) / sx) % (w + tw) - tw
            cy = ((py + vy * t) / sy) % (h + th) - th
            x0, y0 = int(np.floor(cx)), int(np.floor(cy))
            fx, fy = cx - x0, cy - y0
            ys = np.arange(max(0, y0 + 1), min(h, y0 + th))
            xs = np.arange(max(0, x0 + 1), min(w, x0 + tw))
            if len(ys) == 0 or len(xs) == 0:
                continue
            # texture coordinate of output pixel (yy, xx) is (yy - cy, xx - cx)
            ty = ys - y0 - 1
            tx = xs - x0 - 1
            a = tex[np.ix_(ty, tx)]
            b = tex[np.ix_(ty, tx + 1)]
            c = tex[np.ix_(ty + 1, tx)]
            d = tex[np.ix_(ty + 1, tx + 1)]
            gx, gy = 1.0 - fx, 1.0 - fy
            f[np.ix_(ys, xs)] = (a * (1 - gx) * (1 - gy) + b * gx * (1 - gy) + c * (1 - gx) * gy + d * gx * gy)
        f += rng.normal(0.0, 2.0 * scale, size=f.shape)
        out.append(np.clip(np.rint(f), 0, maxv).astype(np.uint16 if bit_depth > 8 else np.uint8))
    return out


def make_sequence(w, h, frames, n_rects=8, vmax=8.0, seed=0, bit_depth=8, chroma="420"):
    """Return a list of frames, each a tuple (Y, U, V) of unsigned sample planes."""
    rng = np.random.default_rng(seed)
    rects = []
    for _ in range(n_rects):
        rw, rh = int(rng.integers(32, 97)), int(rng.integers(32, 97))
        px, py = float(rng.uniform(0, w)), float(rng.uniform(0, h))
        vx = float(rng.integers(-4 * vmax, 4 * vmax + 1)) / 4.0
        vy = float(rng.integers(-4 * vmax, 4 * vmax + 1)) / 4.0
        rects.append((rw, rh, px, py, vx, vy))
    cxs, cys = CHROMA[chroma]
    ys = _plane(rng, w, h, frames, rects, bit_depth, 1, 1)
    us = _plane(rng, w // cxs, h // cys, frames, rects, bit_depth, cxs, cys)
    vs = _plane(rng, w // cxs, h // cys, frames, rects, bit_depth, cxs, cys)
    return list(zip(ys, us, vs))


def to_signed(plane, bit_depth=8):
    """Codec-domain int16 samples: value - 2^(bit_depth-1)."""
    return (plane.astype(np.int32) - (1 << (bit_depth - 1))).astype(np.int16)
