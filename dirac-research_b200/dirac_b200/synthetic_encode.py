"""Encode a seeded synthetic sequence with the device encoder and print timings.

    python -m dirac_b200.synthetic_encode [--width 1920 --height 1080 --frames 32 --reps 2]

Each repetition codes the whole sequence (device-resident input frames) once; the last
repetition runs with per-stage CUDA-event timing.  Default coding parameters are those of
the 1080p workload in bench.py (HD1080P50 GOP, QF 7, DAUB9_7 / DD9_7 depth 4, OBMC 16/12,
quarter-pel).  Useful on its own and as the command under a profiler.
"""
import argparse
import sys
import time


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--frames", type=int, default=32)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--qf", type=float, default=7.0)
    ap.add_argument("--seed", type=int, default=1000)
    a = ap.parse_args(argv)

    import torch

    from . import encoder as E
    from . import synth

    params = dict(cformat=2, width=a.width, height=a.height, luma_depth=8, chroma_depth=8, qf=a.qf, l1_sep=3,
                  num_l1=7, cpd=32.0, xblen=16, yblen=16, xbsep=12, ybsep=12, mv_precision=2, intra_filter=6,
                  inter_filter=0, wlt_depth=4)
    frames = synth.make_sequence(a.width, a.height, a.frames, n_rects=24, vmax=24, seed=a.seed)
    dev = [tuple(torch.from_numpy(p).cuda() for p in fr) for fr in frames]
    st = torch.cuda.Stream()
    enc = E.SequenceEncoder(params, max_pictures=a.frames, stream=st)

    def run():
        enc.reset()
        for f in dev:
            enc.load(f)
        enc.end_sequence()
        while enc.code_next() is not None:
            pass
        st.synchronize()

    for r in range(a.reps):
        last = r == a.reps - 1
        if last:
            enc.profile(True)
        t = time.perf_counter()
        run()
        dt = time.perf_counter() - t
        print(f"rep {r}: {1000 * dt:.1f} ms wall, {a.frames / dt:.1f} frames/s" + (" (profiled)" if last else ""))
    for k, (ms, calls) in enc.profile(False).items():
        print(f"  {k:18s} {ms:9.2f} ms  {calls:4d} calls")
    enc.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
