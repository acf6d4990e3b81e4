#!/usr/bin/env python
"""Benchmark of the Dirac coding hot path on B200: 1080p 4:2:0 8-bit frames/s.

Workload (one "step"): the data-parallel coding loop of the reference encoder over a
32-frame synthetic 1920x1080 4:2:0 8-bit sequence (24 moving textured rectangles, velocities
up to 24 px/frame): GOP of the HD1080P50 preset (L1 separation 3, 7 L1 pictures per GOP),
quality factor 7, DAUB9_7 intra / DD9_7 inter transforms of depth 4, OBMC blocks 16x16 at
separation 12, quarter-pel hierarchical motion estimation with mode decision, motion
compensation, quantiser choice and quantisation, inverse transform and reconstruction, all
bit-exact with the reference.  Arithmetic coding is not part of the path (host code in the
reference); the encoder keeps the initial entropy-correction factors.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gpu|reference]

`value`: frames/s with the input frames resident in HBM.  `e2e`: the same through the
encoder's C ABI from pinned host frames, reading back per picture what the host coder needs
(quantised indices, band choices, code-block skips, motion data).  Every step works on
about 2 GB of distinct device buffers (far above the 126 MB L2), so no L2 flush is needed.
Under torchrun each rank encodes its own sequence (replicas, weak scaling, no collective on
the data path); times are device times, max over ranks.  `--impl reference` times the
reference encoder itself (its public C API) on this host's cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dirac-research_b200"))

METRIC = "1080p frames/s (DWT+ME+OBMC, bit-exact) batched vs plain; p99 latency"
PARAMS = dict(cformat=2, width=1920, height=1080, luma_depth=8, chroma_depth=8, qf=7.0, l1_sep=3, num_l1=7,
              cpd=32.0, xblen=16, yblen=16, xbsep=12, ybsep=12, mv_precision=2, intra_filter=6, inter_filter=0,
              wlt_depth=4)
VIDEO_FORMAT_HD_1080P50 = 14
CPU_SAMPLE_FRAMES = 10


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--frames", type=int, default=32)
    ap.add_argument("--impl", choices=["gpu", "reference"], default="gpu")
    return ap.parse_args()


def workload_name(frames):
    return (f"encode 1920x1080 4:2:0 8-bit, {frames} frames per step (synthetic, 24 rects, v<=24 px/frame); "
            "GOP L1_sep 3 / num_L1 7, QF 7, DAUB9_7 intra / DD9_7 inter depth 4, OBMC 16x16 sep 12, quarter-pel ME; "
            "stages ME+MC+DWT+quantise+IDWT+MC+clip")


def make_frames(frames, seed):
    """8-bit planes [(Y, U, V)] of the synthetic sequence."""
    from dirac_b200 import synth

    return synth.make_sequence(PARAMS["width"], PARAMS["height"], frames, n_rects=24, vmax=24, seed=seed,
                               bit_depth=8, chroma="420")


# ---------------------------------------------------------------------------------------------
# CPU side: the reference encoder (oracle/_ref) for cpu_baseline and --impl reference
# ---------------------------------------------------------------------------------------------

def ref_config():
    cfg = {k: v for k, v in PARAMS.items() if k not in ("luma_depth", "chroma_depth")}
    cfg["video_format"] = VIDEO_FORMAT_HD_1080P50
    return cfg


_WORKER_FRAMES = None


def _init_worker(frames):
    global _WORKER_FRAMES
    _WORKER_FRAMES = frames


def _ref_encode(_):
    """One reference encode of the worker's frames (stock encoder: adaptive entropy factors)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import reference_encode

    t0 = time.perf_counter()
    reference_encode(ref_config(), _WORKER_FRAMES, freeze=False)
    return time.perf_counter() - t0


def reference_available():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Reference

    return Reference.available()


def cpu_baseline_single(frames):
    """The reference encoder in this process (one core) on the first frames of the sequence."""
    global _WORKER_FRAMES
    _WORKER_FRAMES = frames
    _ref_encode(None)  # warm-up (page-in, allocator)
    dt = _ref_encode(None)
    return {"value": len(frames) / dt, "unit": "frames/s", "cores": 1, "kind": "reference",
            "sample": f"reference encoder (dirac_encoder_* API, plain-C build) on the first {len(frames)} frames "
                      f"of the step's sequence: {dt:.2f} s on 1 core"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if not reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libdirac_ref.so was not built "
                          "(the reference sources were absent at build time)"}), flush=True)
        return
    import multiprocessing as mp

    frames = make_frames(CPU_SAMPLE_FRAMES, seed=1000)
    procs = min(os.cpu_count() or 1, 128)  # about 0.5 GB of host memory per encode
    ctx = mp.get_context("spawn")
    walls = []
    with ctx.Pool(procs, initializer=_init_worker, initargs=(frames,)) as pool:
        for k in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            pool.map(_ref_encode, range(procs), chunksize=1)
            dt = time.perf_counter() - t0
            if k >= args.warmup:
                walls.append(dt)
    wall = statistics.median(walls)
    value = procs * CPU_SAMPLE_FRAMES / wall
    sample = (f"{procs} concurrent reference encodes (one per host core) of the first {CPU_SAMPLE_FRAMES} frames "
              f"of the sequence per step; median step {wall:.2f} s")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * wall, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": workload_name(CPU_SAMPLE_FRAMES), "host_processes": procs,
                       "note": "the reference encoder includes its arithmetic coder and bitstream output"},
            "cpu_baseline": {"value": value, "unit": "frames/s", "cores": procs, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# GPU clocks sampled during the timed region
# ---------------------------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.proc = None
        self.device_index = device_index

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device_index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = [r.split(", ") for r in out.strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for name, val in zip(names, r[5:9]):
                if val.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ---------------------------------------------------------------------------------------------

def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    frames = make_frames(args.frames, seed=1000 + rank)
    # CPU baseline first (rank 0, N=1), before any GPU call
    cpu_baseline = None
    if world == 1 and rank == 0:
        if reference_available():
            cpu_baseline = cpu_baseline_single(frames[:CPU_SAMPLE_FRAMES])
        else:
            cpu_baseline = {"value": None, "unit": "frames/s", "cores": 1, "kind": "reference",
                            "sample": "unavailable: oracle/_ref/libdirac_ref.so was not built"}

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    import dirac_b200
    from dirac_b200 import encoder as E
    from dirac_b200.roofline import stage_bytes

    lib = dirac_b200.load()
    stream = torch.cuda.Stream()
    dev_frames = [tuple(torch.from_numpy(p).cuda() for p in fr) for fr in frames]
    torch.cuda.synchronize()
    enc = E.SequenceEncoder(PARAMS, max_pictures=args.frames, stream=stream)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(ms):
        if world > 1:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return ms

    def step(src, events=None, read=None):
        enc.reset()
        for f in src:
            enc.load(f)
        enc.end_sequence()
        infos = []
        while True:
            if events is not None:
                e = torch.cuda.Event(enable_timing=True)
                e.record(stream)
                events.append(e)
            info = enc.code_next()
            if info is None:
                return infos
            infos.append(info)
            if read is not None:
                read(info)

    for _ in range(args.warmup):
        infos = step(dev_frames)
    stream.synchronize()

    # ---- timed region: inputs resident in HBM ------------------------------------------------
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    launches0 = lib.dgpu_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step(dev_frames)
    ev1.record(stream)
    stream.synchronize()
    barrier()
    launches = lib.dgpu_launch_count() - launches0
    clk = clocks.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    ms_per_step = ms / args.steps
    value = world * args.frames * args.steps / (ms / 1000.0)

    # ---- per-picture latency (device timeline, coding order) ---------------------------------
    lat = []
    for _ in range(max(1, args.steps)):
        evs = []
        step(dev_frames, events=evs)
        stream.synchronize()
        lat += [evs[k].elapsed_time(evs[k + 1]) for k in range(len(evs) - 1)]
    lat.sort()
    latency = {"p50": statistics.median(lat), "p99": lat[min(len(lat) - 1, int(round(0.99 * (len(lat) - 1))))],
               "max": lat[-1], "pictures": len(lat)}

    # ---- stage breakdown and the roofline of the dominant stage ------------------------------
    enc.profile(True)
    reps = 2
    for _ in range(reps):
        infos = step(dev_frames)
    prof = enc.profile(False)
    stage_ms = {k: v[0] / reps for k, v in prof.items()}
    alg = stage_bytes(PARAMS, infos)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    dominant = max(stage_ms, key=stage_ms.get)
    per_stage = {k: {"ms_per_step": round(stage_ms[k], 3),
                     "gbs": round(alg[k] / (stage_ms[k] / 1000.0) / 1e9, 1) if stage_ms[k] > 0 else None,
                     "frac": round(alg[k] / (stage_ms[k] / 1000.0) / 1e9 / peak, 4) if stage_ms[k] > 0 else None}
                 for k in stage_ms}
    achieved = alg[dominant] / (stage_ms[dominant] / 1000.0) / 1e9
    roofline = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks
                else "fallback 6650 GB/s (of fallback)",
                "algorithmic_bytes_per_step": alg, "stages": per_stage,
                "note": "stage times from CUDA events on the encoder stream in a separate profiled pass"}

    # ---- end to end through the C ABI with host buffers --------------------------------------
    pinned = [tuple(torch.from_numpy(p).pin_memory() for p in fr) for fr in frames]
    pinned_np = [tuple(t.numpy() for t in fr) for fr in pinned]
    items = [(E.QINDEX, c) for c in range(3)] + [(E.BANDS, c) for c in range(3)] + \
            [(E.CBSKIP, c) for c in range(3)] + [(E.MV, 0), (E.MODE, 0), (E.DC, 0), (E.SPLIT, 0)]
    bufs = {}
    d2h = [0]

    def read(info):
        pn = info["pnum"]
        for what, c in items:
            n = lib.dgpu_encoder_item_bytes(enc.handle, pn, what, c)
            if n == 0:
                continue
            b = bufs.get((what, c, n))
            if b is None:
                b = bufs[(what, c, n)] = torch.empty(n, dtype=torch.uint8, pin_memory=True)
            rc = lib.dgpu_encoder_read(enc.handle, pn, what, c, b.data_ptr(), n, 1)
            if rc:
                raise RuntimeError(f"dgpu_encoder_read failed: {rc}")
            d2h[0] += n

    for _ in range(max(1, args.warmup)):
        step(pinned_np, read=read)
    stream.synchronize()
    barrier()
    d2h[0] = 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step(pinned_np, read=read)
    e1.record(stream)
    stream.synchronize()
    barrier()
    ems = max_over_ranks(e0.elapsed_time(e1))
    h2d = sum(p.nbytes for fr in pinned_np for p in fr)
    e2e = {"value": world * args.frames * args.steps / (ems / 1000.0), "unit": "frames/s",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h[0] // args.steps}
    enc.close()

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
                "config": {"workload": workload_name(args.frames), "frames_per_step": args.frames,
                           "global_batch": world * args.frames, "parallelism": f"replicas{world}",
                           "form": "plain (one sequence per GPU)",
                           "l2": "inputs and working set larger than L2 (no flush needed)"},
                "roofline": roofline, "cpu_baseline": cpu_baseline, "e2e": e2e,
                "latency_ms": latency, "gpu_launches": launches, "clocks": clk}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
