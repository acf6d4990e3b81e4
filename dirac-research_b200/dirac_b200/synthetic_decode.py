"""Code a seeded synthetic sequence with the device encoder, then decode it with the device
decoder and print timings.

    python -m dirac_b200.synthetic_decode [--width 1920 --height 1080 --frames 32 --reps 3]

The decoder's inputs (each picture's quantised indices, band and code-block choices and
motion data, as the encoder produced them) are device-resident; each repetition decodes the
whole sequence in coding order and releases it.  The first line gives the number of library
kernel launches before decoding starts (the encoder's), so that a profiler can skip them.
Coding parameters are those of the 1080p workload in bench.py.
"""
import argparse
import sys


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--frames", type=int, default=32)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=1000)
    a = ap.parse_args(argv)

    import numpy as np
    import torch

    from . import _lib
    from . import decoder as D
    from . import encoder as E
    from . import synth

    params = dict(cformat=2, width=a.width, height=a.height, luma_depth=8, chroma_depth=8, qf=7.0, l1_sep=3,
                  num_l1=7, cpd=32.0, xblen=16, yblen=16, xbsep=12, ybsep=12, mv_precision=2, intra_filter=6,
                  inter_filter=0, wlt_depth=4)
    frames = synth.make_sequence(a.width, a.height, a.frames, n_rects=24, vmax=24, seed=a.seed)
    st = torch.cuda.Stream()
    enc = E.SequenceEncoder(params, max_pictures=a.frames, stream=st)
    infos = enc.encode(frames)
    m = 1 << params["wlt_depth"]
    sizes = [(a.height, a.width), (a.height // 2, a.width // 2), (a.height // 2, a.width // 2)]
    shapes = [tuple((x + m - 1) // m * m for x in s) for s in sizes]
    lib = _lib.load()
    dec = D.SequenceDecoder(D.decoder_params(params), max_pictures=a.frames, stream=st)
    prepared, pnums = [], []
    for info in infos:
        pn = info["pnum"]
        pnums.append(pn)
        q = [torch.from_numpy(enc.read(pn, E.QINDEX, c).reshape(shapes[c])).cuda() for c in range(3)]
        cbs = torch.from_numpy(np.concatenate([enc.read(pn, E.CBSKIP, c) for c in range(3)])).cuda()
        refs = [] if info["intra"] else [x for x in (info["ref1"], info["ref2"]) if x >= 0]
        mot = None
        if not info["intra"]:
            mv = enc.read(pn, E.MV).reshape(info["num_refs"], -1, 2)
            mot = {"mv": [torch.from_numpy(np.ascontiguousarray(mv[k])).cuda() for k in range(len(refs))],
                   **{k: torch.from_numpy(enc.read(pn, w)).cuda() for k, w in (("mode", E.MODE), ("dc", E.DC),
                                                                                ("split", E.SPLIT))}}
        prepared.append(dec.prepare(pn, info["intra"], refs, info["filter"], q,
                                    [enc.read(pn, E.BANDS, c) for c in range(3)], cbs, mot))
    st.synchronize()
    print(f"launches before decoding: {lib.dgpu_launch_count()}")
    for r in range(a.reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for p in prepared:
            dec.decode_prepared(p)
        e1.record(st)
        for pn in pnums:
            dec.release(pn)
        st.synchronize()
        ms = e0.elapsed_time(e1)
        print(f"rep {r}: {ms:.2f} ms device, {len(prepared) / (ms / 1000.0):.1f} frames/s")
    dec.close()
    enc.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
