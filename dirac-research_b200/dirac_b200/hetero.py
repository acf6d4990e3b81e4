"""The heterogeneous picture-batch workload: 64 pictures per batch from the synthetic generator
in mixed sizes, formats and bit depths -- 16 x 352x288 4:2:0 8-bit, 16 x 720x576 4:2:0
8-bit, 16 x 1280x720 4:2:0 10-bit (16-bit storage), 16 x 1920x1080 4:2:2 10-bit -- each with
a random transform filter from {Haar, LeGall (5,3), Deslauriers-Dubuc (13,7), Fidelity (the
reference codes it as Daubechies (9,7)), Daubechies (9,7)} and a random depth in 3..5.
Pictures alternate between one reference (P) and two (B); their motion data comes from the
library's motion estimation against the neighbouring frames of their class's sequence, so
that motion compensation works on real vectors and modes."""
import numpy as np
import torch

from . import _lib, synth
from .motion import MotionEstimator

# (width, height, chroma, bits, OBMC blocks (xblen, yblen, xbsep, ybsep))
CLASSES = [
    (352, 288, "420", 8, (12, 12, 8, 8)),
    (720, 576, "420", 8, (12, 12, 8, 8)),
    (1280, 720, "420", 10, (16, 16, 12, 12)),
    (1920, 1080, "422", 10, (16, 16, 12, 12)),
]
CFORMAT = {"444": 0, "422": 1, "420": 2}
# Haar (either shift), LeGall (5,3), Deslauriers-Dubuc (13,7), Fidelity, Daubechies (9,7)
FILTER_CHOICES = [(3, 4), (1,), (2,), (5,), (6,)]
ME_LAMBDA = 10.0  # the encoder's motion-estimation lambda at quality factor 7


def block_params(w, h, blk, precision=2):
    xbl, ybl, xbs, ybs = blk
    return _lib.BlockParams(precision=precision, xblen=xbl, yblen=ybl, xbsep=xbs, ybsep=ybs,
                            xnum_sb=(w + 4 * xbs - 1) // (4 * xbs), ynum_sb=(h + 4 * ybs - 1) // (4 * ybs))


def make_inputs(per_class=16, seed=11, qf=7.0, cpd=32.0):
    """Returns (pictures, motion, planes, refs): the dgpu_batch_picture dicts, the motion dicts
    (CUDA tensors), each picture's three int16 codec-sample planes as CUDA tensors, and the
    reference tensors kept alive for the batch."""
    rng = np.random.default_rng(seed)
    pictures, motion, planes, keep = [], [], [], []
    for ci, (w, h, chroma, bits, blk) in enumerate(CLASSES):
        seq = synth.make_sequence(w, h, per_class + 2, n_rects=max(4, w // 80), vmax=8, seed=seed * 10 + ci,
                                  bit_depth=bits, chroma=chroma)
        dev = [[torch.from_numpy(synth.to_signed(p, bits)).cuda() for p in f] for f in seq]
        keep.append(dev)
        bp = block_params(w, h, blk)
        tasks = []
        for k in range(per_class):
            two = k % 2 == 1
            tasks.append((k + 1, k, k + 2 if two else -1, ME_LAMBDA))
        est = MotionEstimator(bp, CFORMAT[chroma], bits).EstimateBatch(dev, tasks)
        for k, (cur, r1, r2, _) in enumerate(tasks):
            e = est[k]
            nref = 2 if r2 >= 0 else 1
            filt = int(rng.choice(FILTER_CHOICES[int(rng.integers(len(FILTER_CHOICES)))]))
            depth = int(rng.integers(3, 6))
            ratio = float((e["mode"] == 0).sum().item()) / e["mode"].numel()
            pictures.append(dict(cformat=CFORMAT[chroma], width=w, height=h, luma_depth=bits, chroma_depth=bits,
                                 filter=filt, wlt_depth=depth, intra=0, is_b=int(nref == 2), qf=qf, cpd=cpd,
                                 intra_ratio=ratio, bp=bp))
            motion.append({"ref1": dev[r1], "ref2": dev[r2] if nref == 2 else None, "mv1": e["mv"][0].contiguous(),
                           "mv2": e["mv"][1].contiguous() if nref == 2 else None, "mode": e["mode"],
                           "dc": e["dc"], "split": e["split"]})
            planes.append([t.clone() for t in dev[cur]])
    return pictures, motion, planes, keep


def stage_bytes(pictures):
    """Algorithmic bytes of one batch run by stage (pre: reference upconversions, motion
    compensation SUBTRACT and forward transforms; quant: 16 B per coefficient; post: inverse
    transforms and motion compensation ADD with the clip), counting every byte once."""
    from .roofline import dwt_bytes

    pre = quant = post = 0
    for p in pictures:
        xs = 0 if p["cformat"] == 0 else 1
        ys = 1 if p["cformat"] == 2 else 0
        comps = [(p["width"], p["height"]), (p["width"] >> xs, p["height"] >> ys),
                 (p["width"] >> xs, p["height"] >> ys)]
        mul = 1 << p["wlt_depth"]
        pad = [((a + mul - 1) // mul * mul, (b + mul - 1) // mul * mul) for a, b in comps]
        samples = sum(a * b for a, b in comps)
        d = sum(dwt_bytes(a, b, p["wlt_depth"]) for a, b in pad)
        nref = 0 if p["intra"] else (2 if p.get("is_b") else 1)
        mc = samples * (4 + 8 * nref) if nref else samples * 4
        pre += d + (mc if nref else 0)
        post += d + mc
        quant += 16 * sum(a * b for a, b in pad)
    return {"pre": pre, "quant": quant, "post": post}


def upconvert_bytes(motion):
    """10 B per sample of every distinct reference plane (2 B read, 8 B written)."""
    seen = {}
    for m in motion:
        if m is None:
            continue
        for key in ("ref1", "ref2"):
            if m.get(key) is None:
                continue
            for t in m[key]:
                seen[t.data_ptr()] = t.numel()
    return 10 * sum(seen.values())


def main(argv=None):
    """python -m dirac_b200.hetero [--runs N]: builds the workload, codes it N times and prints
    the wall time per run and one run's stage times (also the command for profiling)."""
    import argparse
    import time

    from .batch import PictureBatch

    ap = argparse.ArgumentParser()
    ap.add_argument("--runs", type=int, default=4)
    a = ap.parse_args(argv)
    pictures, motion, planes, keep = make_inputs()
    batch = PictureBatch(pictures, motion)
    for r in range(a.runs):
        for k in range(len(planes)):
            batch.load(k, planes[k])
        torch.cuda.synchronize()
        t = time.perf_counter()
        batch.run()
        torch.cuda.synchronize()
        print(f"run {r}: {1000 * (time.perf_counter() - t):.2f} ms for {len(pictures)} pictures")
    print("stage ms (pre, quant, post):", [round(x, 3) for x in batch.stage_times()])
    batch.close()
    del keep
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
