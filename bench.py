#!/usr/bin/env python
"""Benchmark of the Dirac coding hot path on B200: 1080p 4:2:0 8-bit frames/s.

Workload (one "step"): the data-parallel coding loop of the reference encoder over a
32-frame synthetic 1920x1080 4:2:0 8-bit sequence (24 moving textured rectangles, velocities
up to 24 px/frame): GOP of the HD1080P50 preset (L1 separation 3, 7 L1 pictures per GOP),
quality factor 7, DAUB9_7 intra / DD9_7 inter transforms of depth 4, OBMC blocks 16x16 at
separation 12, quarter-pel hierarchical motion estimation with mode decision, motion
compensation, quantiser choice and quantisation, inverse transform and reconstruction, all
bit-exact with the reference.  `value` keeps the initial entropy-correction factors (the device
work of the path alone); `e2e` codes every picture's subbands on the host and adapts the factors
from the coded bytes, so its quantiser choices, and its locally decoded pictures, are the stock
reference encoder's (checked against the reference's own run of the same sequence in
`parity_vs_reference`).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gpu|reference]

`value`: frames/s of the batched form (--streams sequences per GPU, each with its own
encoder, CUDA stream and host thread, split into --me-groups encoder groups that run
concurrently: each group's motion estimation is one batched launch, and one group's
estimation overlaps another's coding) with the input frames resident in HBM;
`batched_one_group` gives the same with all sequences in one group, `batched_streams_only`
without groups (each sequence estimating alone), `plain` for one sequence at a time.
`e2e`: the batched form through
the encoder's C ABI from pinned host frames, reading back per picture what the host coder
needs (quantised indices, band choices, code-block skips, motion data) and arithmetic-coding
the subbands on the host threads (`e2e_hot_path`: the same without the host coder).  Every step works on
gigabytes of distinct device buffers (far above the 126 MB L2), so no L2 flush is needed.
`decoding`: the plain form's coded sequence decoded by the device decoder (dequantisation,
inverse transform, motion compensation, clip, output samples), its output checked against the
encoder's local decode.
Under torchrun each rank encodes its own sequence (replicas, weak scaling, no collective on
the data path); times are device times, max over ranks.  `--impl reference` times the
reference encoder itself (its public C API) on this host's cores.
"""
import argparse
import json
import os
import resource

import numpy as np
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dirac-research_b200"))

METRIC = "1080p frames/s (DWT+ME+OBMC, bit-exact) batched vs plain; p99 latency"
PARAMS = dict(cformat=2, width=1920, height=1080, luma_depth=8, chroma_depth=8, qf=7.0, l1_sep=3, num_l1=7,
              cpd=32.0, xblen=16, yblen=16, xbsep=12, ybsep=12, mv_precision=2, intra_filter=6, inter_filter=0,
              wlt_depth=4)
VIDEO_FORMAT_HD_1080P50 = 14
REF_WARMUP_FRAMES = 2  # a reference warm-up encode (page-in, allocator): the sequence's first frames
# the encoder's streaming stages and the kernels each one runs
STREAMING_KERNELS = {"dwt_forward": "dwt_forward_fast_kernel / dwt_forward_level_kernel",
                     "dwt_inverse": "dwt_inverse_fast_kernel / dwt_inverse_level_kernel",
                     "mc_subtract": "obmc_kernel (SUBTRACT)", "mc_add_clip": "obmc_kernel (ADD, clip fused)",
                     "upconvert": "upconvert_kernel",
                     "quantisation": "band_max, stats, seq_resolve, gather_stats, quantise, dc_intra kernels "
                                     "and the host Lagrangian"}
# motion-estimation kernel classes of dgpu_me_profile and counters of dgpu_debug_wavefront
ME_CLASSES = {"pel_search": (1, 2), "subpel_refinement": (3,), "mode_decision": (4, 5)}
ME_OP_INDEX = {"pel_search": 0, "subpel_refinement": 1, "mode_decision": 2}
# DRAM bytes per algorithmic operation of each motion-estimation kernel, from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum over the launch's counted operations) of the
# 13-frame encode leg: sub-pel refinement 207.08 MB read + 4.97 MB written over 4378228940
# operations; the bench's launches are scaled from it by their operation counts
ME_TRAFFIC_PER_OP = {"subpel_refinement": (207.08e6 + 4.97e6) / 4378228940}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--frames", type=int, default=32)
    ap.add_argument("--streams", type=int, default=12, help="concurrent sequences per GPU (batched form)")
    ap.add_argument("--me-occupancy", type=int, default=8,
                    help="resident CTAs per SM of the motion-estimation wavefront kernels (1-8)")
    ap.add_argument("--me-unit-life", type=int, default=0,
                    help="units a motion-estimation wavefront warp takes before it exits (0: persistent)")
    ap.add_argument("--lane-priority", type=int, default=0,
                    help="CUDA stream priority of the sequences' coding streams (negative: above the encoder "
                         "groups' estimation streams, which run at the default 0)")
    ap.add_argument("--blocking-waits", type=int, default=0,
                    help="the library's host waits for the device: 0 poll, 1 sleep on blocking-sync events "
                         "(measured slower: the plain form loses a third), 2 poll and yield (measured no faster)")
    ap.add_argument("--me-groups", type=int, default=3,
                    help="encoder groups the batched form's sequences are split into (run concurrently)")
    ap.add_argument("--double-buffer", type=int, default=0,
                    help="1: each group alternates two sets of sequences, one set's estimation running "
                         "while the other set is coded (measured slower: the sets contend for the device)")
    ap.add_argument("--serving-rate", type=float, default=40.0, help="stream arrivals per second (Poisson)")
    ap.add_argument("--serving-seconds", type=float, default=6.0,
                    help="length of the serving-loop run reported under 'serving' (0: skip)")
    ap.add_argument("--hetero-steps", type=int, default=5,
                    help="timed runs of the heterogeneous 64-picture batch reported under 'heterogeneous_batch' "
                         "(0: skip)")
    ap.add_argument("--decode", type=int, default=1,
                    help="1: report the device decoder on the plain form's coded sequence under 'decoding'")
    ap.add_argument("--cpu-baseline", type=int, default=1,
                    help="1: time the reference encoder on this host first (cpu_baseline, parity_vs_reference)")
    ap.add_argument("--leg", choices=["all", "encode", "decode"], default="all",
                    help="encode / decode: only the plain form's coding (or its device decoding) of the sequence, "
                         "--warmup then --steps times, for profilers; prints the launch count, no bench line")
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


def _ref_encode(nframes, keep=None):
    """One reference encode of the worker's first nframes frames (stock encoder: adaptive
    entropy factors); with keep (a list), (locally decoded frames, bitstream) is appended."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import reference_encode, reference_encode_stream

    frames = _WORKER_FRAMES[:nframes]
    t0 = time.perf_counter()
    if keep is None:
        reference_encode(ref_config(), frames, freeze=False)
    else:
        rec, _, stream = reference_encode_stream(ref_config(), frames, freeze=False)
        keep.append((rec, stream))
    return time.perf_counter() - t0


def reference_available():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Reference

    return Reference.available()


def cpu_baseline_single(frames, keep=None):
    """The reference encoder in this process (one core) on the whole sequence; with keep (a
    list), the encode's (locally decoded frames, bitstream) is appended there."""
    global _WORKER_FRAMES
    _WORKER_FRAMES = frames
    _ref_encode(REF_WARMUP_FRAMES)  # warm-up (page-in, allocator)
    dt = _ref_encode(len(frames), keep)
    return {"value": len(frames) / dt, "unit": "frames/s", "cores": 1, "kind": "reference",
            "sample": f"reference encoder (dirac_encoder_* API, plain-C build, stock adaptive entropy factors, its "
                      f"arithmetic coding and bitstream output included) on the step's whole {len(frames)}-frame "
                      f"sequence: {dt:.2f} s on 1 core"}


def cpu_decode_baseline(stream, nframes):
    """The reference decoder in this process (one core) on the reference encoder's bitstream of
    the first frames of the sequence."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import reference_decode

    w, h = PARAMS["width"], PARAMS["height"]
    reference_decode(stream, w, h, PARAMS["cformat"], nframes)  # warm-up
    t0 = time.perf_counter()
    out = reference_decode(stream, w, h, PARAMS["cformat"], nframes)
    dt = time.perf_counter() - t0
    n = sum(f is not None for f in out)
    return {"value": n / dt, "unit": "frames/s", "cores": 1, "kind": "reference",
            "sample": f"reference decoder (dirac_decoder_* API, plain-C build) on the reference encoder's bitstream "
                      f"of the first {nframes} frames of the sequence ({len(stream)} bytes): {n} frames in "
                      f"{dt:.2f} s on 1 core, its arithmetic decoding included"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if not reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libdirac_ref.so was not built "
                          "(the reference sources were absent at build time)"}), flush=True)
        return
    import multiprocessing as mp

    frames = make_frames(args.frames, seed=1000)
    procs = min(os.cpu_count() or 1, 128)  # about 0.5 GB of host memory per encode
    ctx = mp.get_context("spawn")
    walls = []
    with ctx.Pool(procs, initializer=_init_worker, initargs=(frames,)) as pool:
        for k in range(args.warmup + args.steps):
            n = REF_WARMUP_FRAMES if k < args.warmup else args.frames
            t0 = time.perf_counter()
            pool.map(_ref_encode, [n] * procs, chunksize=1)
            dt = time.perf_counter() - t0
            if k >= args.warmup:
                walls.append(dt)
    wall = statistics.median(walls)
    value = procs * args.frames / wall
    sample = (f"{procs} concurrent reference encodes (one per host core) of the whole {args.frames}-frame sequence "
              f"per step (warm-up steps: its first {REF_WARMUP_FRAMES} frames); median step {wall:.2f} s")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * wall, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": workload_name(args.frames), "host_processes": procs,
                       "note": "the stock reference encoder, its arithmetic coding and bitstream output included"},
            "cpu_baseline": {"value": value, "unit": "frames/s", "cores": procs, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# multi-rank helpers (one process per GPU; replicas, no collective on the data path)
# ---------------------------------------------------------------------------------------------

def max_over_ranks_ms(ms, world, device):
    """The slowest rank's time: every rank calls this with its own device time."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, units_per_rank_step, steps, ms):
    """Units per second of the whole job: every rank's units over the slowest rank's time."""
    return world * units_per_rank_step * steps / (ms / 1000.0)


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
# heterogeneous picture batch (the batched launch of 64 mixed pictures)
# ---------------------------------------------------------------------------------------------

def run_hetero(args, peak, peaks):
    """64 pictures (16 each of CIF 8-bit, 576p 8-bit, 720p 10-bit 4:2:0, 1080p 10-bit 4:2:2) with
    random filters and depths: motion compensation SUBTRACT, forward transform, quantisation,
    inverse transform, motion compensation ADD per picture, in one batch (CUDA graphs around
    the host quantiser choice).  Device-resident inputs for `value`; `e2e` loads every picture
    from pinned host memory and reads its quantised indices back each step."""
    import torch

    from dirac_b200 import hetero as H
    from dirac_b200.batch import QINDEX, PictureBatch

    pictures, motion, planes, keep = H.make_inputs()
    n = len(pictures)
    batch = PictureBatch(pictures, motion)
    st = torch.cuda.current_stream()

    def step(src, reads=None):
        for k in range(n):
            batch.load(k, src[k])
        batch.run()
        if reads is not None:
            for k in range(n):
                for c in range(3):
                    buf = reads[k][c]
                    batch.lib.dgpu_batch_read(batch.handle, k, QINDEX, c, buf.data_ptr(), buf.numel() * 4, 1)

    def timed(src, steps, reads=None):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            step(src, reads)
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    for _ in range(max(3, args.warmup)):
        step(planes)
    launches0 = batch.lib.dgpu_launch_count()
    ms = timed(planes, args.hetero_steps)
    launches = (batch.lib.dgpu_launch_count() - launches0) // args.hetero_steps
    host = [[t.cpu().pin_memory() for t in pl] for pl in planes]
    host_np = [[t.numpy() for t in pl] for pl in host]
    reads = []
    for k in range(n):
        reads.append([torch.empty(batch.lib.dgpu_batch_item_bytes(batch.handle, k, QINDEX, c) // 4,
                                  dtype=torch.int32, pin_memory=True) for c in range(3)])
    step(host_np, reads)
    ems = timed(host_np, args.hetero_steps, reads)
    stage_ms = [0.0, 0.0, 0.0]
    reps = 3
    for _ in range(reps):
        t = batch.stage_times()
        stage_ms = [a + b / reps for a, b in zip(stage_ms, t)]
    alg = H.stage_bytes(pictures)
    alg["pre"] += H.upconvert_bytes(motion)
    stages = {}
    for name, t in zip(("pre", "quant", "post"), stage_ms):
        gbs = alg[name] / (t / 1000.0) / 1e9
        stages[name] = {"ms": round(t, 3), "algorithmic_bytes": alg[name], "gbs": round(gbs, 1),
                        "frac": round(gbs / peak, 4)}
    h2d = sum(a.nbytes for pl in host_np for a in pl)
    d2h = sum(b.numel() * 4 for r in reads for b in r)
    out = {"value": n * args.hetero_steps / (ms / 1000.0), "unit": "pictures/s", "pictures_per_step": n,
           "ms_per_step": ms / args.hetero_steps, "steps": args.hetero_steps,
           "e2e": {"value": n * args.hetero_steps / (ems / 1000.0), "unit": "pictures/s",
                   "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
           "stages": stages, "gpu_launches_per_step": launches,
           "workload": "16x 352x288 4:2:0 8-bit, 16x 720x576 4:2:0 8-bit, 16x 1280x720 4:2:0 10-bit, "
                       "16x 1920x1080 4:2:2 10-bit; random filter (Haar, LeGall, DD13_7, Fidelity, DAUB9_7) "
                       "and depth 3-5; P and B pictures with motion from the library's estimation; QF 7",
           "note": "stages timed in a separate pass with CUDA events on the batch stream; 'pre' = reference "
                   "upconversions + motion compensation SUBTRACT + forward transforms (one CUDA graph), "
                   "'quant' = quantiser choice (host Lagrangian) + quantisation, 'post' = inverse transforms + "
                   "motion compensation ADD with the clip (one CUDA graph)"}
    batch.close()
    del keep
    return out


def host_band_coding(pictures, depth, ncb):
    """Throughput of the host arithmetic coder (dgpu_code_bands_host, every band of a picture in
    parallel on the library's host threads) over coded pictures [(intra, qindex planes, band
    tables, code-block flags)]: pictures/s and bytes per picture."""
    from dirac_b200.entropy import code_bands

    def run():
        total = 0
        for intra, q, bands, cbs in pictures:
            data, _ = code_bands([intra] * 3, [depth] * 3, q, bands, [ncb] * 3, cbs)
            total += data.size
        return total

    run()  # warm-up (host threads, allocator)
    t0 = time.perf_counter()
    total = run()
    dt = time.perf_counter() - t0
    return {"value": len(pictures) / dt, "unit": "pictures/s", "bytes_per_picture": total / len(pictures),
            "host_threads": min(16, os.cpu_count() or 1),
            "form": "the subbands of the plain form's coded 1080p pictures arithmetic-coded on the host "
                    "(bytes equal to the reference's band coders'), one call per picture"}


def run_decoding(args, enc, infos, peak, cpu_decode=None):
    """The decoding leg: the 1080p sequence the plain form coded, decoded by the device decoder
    (dgpu_decoder_*) from its quantised indices, band and code-block choices and motion data, in
    coding order; every picture's output samples checked against the encoder's locally decoded
    ones.  Device-resident inputs for `value`; page-locked host inputs and output samples read
    back to page-locked host memory for `e2e`.  The CPU baseline is the reference decoder on one
    host core (cpu_decode, measured before any GPU work), with the oracle's restatement of the
    decoder timed beside it."""
    import numpy as np
    import torch

    from dirac_b200 import decoder as D
    from dirac_b200 import encoder as E
    from dirac_b200.roofline import decode_bytes

    st = torch.cuda.current_stream()
    dec = D.SequenceDecoder(D.decoder_params(PARAMS), max_pictures=len(infos), stream=st)
    lib = dec.lib
    m = 1 << PARAMS["wlt_depth"]
    sizes = [(PARAMS["height"], PARAMS["width"]), (PARAMS["height"] // 2, PARAMS["width"] // 2)]
    shapes = [tuple((x + m - 1) // m * m for x in sizes[min(c, 1)]) for c in range(3)]
    dev, host, want, pnums, coded = [], [], [], [], []
    keep = []
    h2d = 0
    n16 = 0  # pictures sent with int16 indices
    for info in infos:
        pn = info["pnum"]
        pnums.append(pn)
        q = [enc.read(pn, E.QINDEX, c).reshape(shapes[c]) for c in range(3)]
        # a picture whose indices all fit 16 bits goes as int16 (index_bits 16): half the bytes
        qin = q
        if all(int(np.abs(a).max()) <= 32767 for a in q):
            qin = [a.astype(np.int16) for a in q]
            n16 += 1
        bands = [enc.read(pn, E.BANDS, c) for c in range(3)]
        cbs = np.concatenate([enc.read(pn, E.CBSKIP, c) for c in range(3)])
        refs = [] if info["intra"] else [x for x in (info["ref1"], info["ref2"]) if x >= 0]
        mot = None
        if not info["intra"]:
            mv = enc.read(pn, E.MV).reshape(info["num_refs"], -1, 2)
            mot = {"mv": [mv[k] for k in range(len(refs))], "mode": enc.read(pn, E.MODE), "dc": enc.read(pn, E.DC),
                   "split": enc.read(pn, E.SPLIT)}
        want.append([enc.read(pn, E.OUTPUT, c) for c in range(3)])
        coded.append((info["intra"], q, bands, [enc.read(pn, E.CBSKIP, c) for c in range(3)]))
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
        hq, hc = [pin(a) for a in qin], pin(cbs)
        hm = None if mot is None else {"mv": [pin(v) for v in mot["mv"]],
                                       **{k: pin(mot[k]) for k in ("mode", "dc", "split")}}
        keep += [hq, hc, hm]
        h2d += sum(t.numel() * t.element_size() for t in hq) + hc.numel()
        if hm is not None:
            h2d += sum(t.numel() * t.element_size() for t in hm["mv"]) + sum(
                hm[k].numel() * hm[k].element_size() for k in ("mode", "dc", "split"))
        np_m = None if hm is None else {"mv": [t.numpy() for t in hm["mv"]],
                                        **{k: hm[k].numpy() for k in ("mode", "dc", "split")}}
        host.append(dec.prepare(pn, info["intra"], refs, info["filter"], [t.numpy() for t in hq], bands,
                                hc.numpy(), np_m))
        dm = None if hm is None else {"mv": [t.cuda() for t in hm["mv"]],
                                      **{k: hm[k].cuda() for k in ("mode", "dc", "split")}}
        dev.append(dec.prepare(pn, info["intra"], refs, info["filter"], [t.cuda() for t in hq], bands, hc.cuda(),
                               dm))
    n_out = [a.size for a in want[0]]
    out_dev = [torch.empty(n, dtype=torch.uint8, device="cuda") for n in n_out]
    out_host = [[torch.empty(n, dtype=torch.uint8, pin_memory=True) for n in n_out] for _ in infos]
    d2h = sum(n_out) * len(infos)

    def step(inputs, read=False):
        for k, I in enumerate(inputs):
            dec.decode_prepared(I)
            if read:
                for c in range(3):
                    rc = lib.dgpu_decoder_read(dec.handle, pnums[k], E.OUTPUT, c, out_dev[c].data_ptr(), n_out[c], 0)
                    if rc:
                        raise RuntimeError(f"dgpu_decoder_read: {rc}")
                    out_host[k][c].copy_(out_dev[c], non_blocking=True)
        for pn in pnums:
            dec.release(pn)

    def timed(inputs, steps, read=False):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            step(inputs, read)
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    for _ in range(max(3, args.warmup)):
        step(dev)
    step(host, read=True)
    launches0 = lib.dgpu_launch_count()
    ms = timed(dev, args.steps)
    launches = (lib.dgpu_launch_count() - launches0) // args.steps
    ems = timed(host, args.steps, read=True)
    matches = all(np.array_equal(out_host[k][c].numpy(), want[k][c]) for k in range(len(infos)) for c in range(3))
    alg = decode_bytes(PARAMS, infos, n16)
    total_alg = sum(alg.values())
    achieved = total_alg * args.steps / (ms / 1000.0) / 1e9
    dec.close()
    del keep

    # CPU baseline: the oracle's restatement of the decoder on the first pictures in coding order
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from dirac_b200 import quant
    from oracle_decoder import decode_picture

    ncb = quant.code_blocks(PARAMS["wlt_depth"], PARAMS["width"], PARAMS["height"])
    cfg = dict(PARAMS)
    done, t_cpu = {}, 0.0
    for k, info in enumerate(infos):
        pn = info["pnum"]
        qn = [enc.read(pn, E.QINDEX, c).reshape(shapes[c]) for c in range(3)]
        b = [np.asarray(x).reshape(-1, 3) for x in [enc.read(pn, E.BANDS, c) for c in range(3)]]
        cb = [enc.read(pn, E.CBSKIP, c) for c in range(3)]
        pic = {"intra": info["intra"], "filter": info["filter"], "qindex": qn, "qidx": [x[:, 0] for x in b],
               "skip": [x[:, 1] for x in b], "cb_skip": cb}
        refs = None
        if not info["intra"]:
            mv = enc.read(pn, E.MV).reshape(info["num_refs"], -1, 2)
            pic["me"] = {"mv": [mv[j] for j in range(info["num_refs"])], "mode": enc.read(pn, E.MODE),
                         "dc": enc.read(pn, E.DC), "split": enc.read(pn, E.SPLIT)}
            refs = [done[x] for x in (info["ref1"], info["ref2"]) if x >= 0]
        t0 = time.perf_counter()
        done[pn] = decode_picture(cfg, pic, refs, ncb)
        t_cpu += time.perf_counter() - t0
        if t_cpu > 10.0 or k + 1 >= 8:
            break
    ncpu = len(done)
    try:
        coding = host_band_coding(coded, PARAMS["wlt_depth"], ncb)
    except Exception as e:  # the coder's measurement must not cost the decoding line
        coding = {"error": repr(e)}
    port = {"value": ncpu / t_cpu, "unit": "frames/s", "cores": 1, "kind": "port",
            "sample": f"the oracle's plain-C restatement of the decoder (dequantisation, inverse transform, motion "
                      f"compensation, clip) on the first {ncpu} pictures in coding order: {t_cpu:.2f} s on 1 core"}
    baseline = cpu_decode if cpu_decode and cpu_decode.get("value") else port
    return {"value": len(infos) * args.steps / (ms / 1000.0), "unit": "frames/s", "frames_per_step": len(infos),
            "ms_per_step": ms / args.steps, "steps": args.steps,
            "e2e": {"value": len(infos) * args.steps / (ems / 1000.0), "unit": "frames/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "output_matches_encoder": bool(matches), "gpu_launches_per_step": launches,
            "int16_index_pictures": n16,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4),
                         "algorithmic_bytes_per_step": alg},
            "cpu_baseline": baseline, "cpu_port": port, "host_band_coding": coding,
            "workload": "decode of the plain form's coded 1920x1080 4:2:0 8-bit 32-picture sequence from its "
                        "quantised indices (int16 where a picture's indices fit, else int32), band and code-block "
                        "choices and motion data; output 8-bit samples"}


def run_leg(args):
    """One leg alone for profilers (ncu's launch lists and captures): the device encoder coding
    the sequence from device-resident frames (encode), or additionally the device decoder
    decoding the coded sequence (decode), --warmup untimed then --steps more times."""
    import torch

    import dirac_b200
    from dirac_b200 import encoder as E
    from dirac_b200.decoder import SequenceDecoder, decoder_params

    lib = dirac_b200.load()
    frames = [tuple(torch.from_numpy(p).cuda() for p in fr) for fr in make_frames(args.frames, seed=1000)]
    enc = E.SequenceEncoder(PARAMS, max_pictures=args.frames)

    def encode():
        enc.reset()
        for f in frames:
            enc.load(f)
        enc.end_sequence()
        out = []
        while True:
            info = enc.code_next()
            if info is None:
                return out
            out.append(info)

    if args.leg == "encode":
        for _ in range(args.warmup):
            encode()
        torch.cuda.synchronize()
        n0 = lib.dgpu_launch_count()
        for _ in range(args.steps):
            encode()
        torch.cuda.synchronize()
        print(json.dumps({"leg": "encode", "launches_per_step": (lib.dgpu_launch_count() - n0) // max(1, args.steps)}))
        return
    infos = encode()
    dec = SequenceDecoder(decoder_params(PARAMS), max_pictures=args.frames)
    inputs = []
    depth = PARAMS["wlt_depth"]
    mul = 1 << depth
    shapes = [(((PARAMS["height"] >> (c > 0)) + mul - 1) // mul * mul,
               ((PARAMS["width"] >> (c > 0)) + mul - 1) // mul * mul) for c in range(3)]
    for info in infos:
        pn = info["pnum"]
        refs = [] if info["intra"] else [x for x in (info["ref1"], info["ref2"]) if x >= 0]
        mot = None
        if not info["intra"]:
            mv = enc.read(pn, E.MV).reshape(info["num_refs"], -1, 2)
            mot = {"mv": [torch.from_numpy(mv[k].copy()).cuda() for k in range(len(refs))],
                   **{k: torch.from_numpy(enc.read(pn, w)).cuda() for k, w in (("mode", E.MODE), ("dc", E.DC),
                                                                                 ("split", E.SPLIT))}}
        q = [enc.read(pn, E.QINDEX, c).reshape(shapes[c]) for c in range(3)]
        if all(int(np.abs(a).max()) <= 32767 for a in q):  # int16 indices, as the decoding leg sends them
            q = [a.astype(np.int16) for a in q]
        q = [torch.from_numpy(a).cuda() for a in q]
        cbs = torch.from_numpy(np.concatenate([enc.read(pn, E.CBSKIP, c) for c in range(3)])).cuda()
        inputs.append((pn, dec.prepare(pn, info["intra"], refs, info["filter"], q,
                                       [enc.read(pn, E.BANDS, c) for c in range(3)], cbs, mot)))

    def decode():
        for _, I in inputs:
            dec.decode_prepared(I)
        for pn, _ in inputs:
            dec.release(pn)

    for _ in range(args.warmup):
        decode()
    torch.cuda.synchronize()
    n0 = lib.dgpu_launch_count()
    for _ in range(args.steps):
        decode()
    torch.cuda.synchronize()
    print(json.dumps({"leg": "decode", "launches_per_step": (lib.dgpu_launch_count() - n0) // max(1, args.steps)}))


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.leg != "all":
        run_leg(args)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    frames = make_frames(args.frames, seed=1000 + rank)
    # CPU baseline first (rank 0, N=1), before any GPU call
    cpu_baseline = None
    cpu_decode = None
    ref_recon = None  # the reference encoder's locally decoded pictures of this sequence
    if world == 1 and rank == 0 and args.cpu_baseline:
        if reference_available():
            keep = []
            cpu_baseline = cpu_baseline_single(frames, keep)
            ref_recon = keep[0][0]
            if args.decode:
                try:
                    cpu_decode = cpu_decode_baseline(keep[0][1], args.frames)
                except Exception as e:  # the decoding leg falls back to the oracle's decoder
                    cpu_decode = {"error": repr(e)}
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

    import ctypes

    import numpy as np

    import dirac_b200
    from dirac_b200 import encoder as E
    from dirac_b200.adaptive import AdaptiveCoder
    from dirac_b200.roofline import stage_bytes

    lib = dirac_b200.load()
    dev_frames = [tuple(torch.from_numpy(p).cuda() for p in fr) for fr in frames]
    pinned = [tuple(torch.from_numpy(p).pin_memory() for p in fr) for fr in frames]
    pinned_np = [tuple(t.numpy() for t in fr) for fr in pinned]
    torch.cuda.synchronize()
    from dirac_b200.adaptive import CODED_ITEMS as items

    class Lane:
        """One sequence encoder on its own CUDA stream (the batched form runs several, each
        driven by its own host thread)."""

        def __init__(self):
            self.stream = torch.cuda.Stream(priority=args.lane_priority)
            self.enc = E.SequenceEncoder(PARAMS, max_pictures=args.frames, stream=self.stream)
            self.bufs = {}
            self.d2h = 0
            self.coder = AdaptiveCoder(self.enc, PARAMS)
            self.pictures = 0

        def read(self, info):
            """The coded picture's results the host coder needs, into page-locked buffers
            (reused picture after picture); returns numpy views by (item, component)."""
            pn = info["pnum"]
            got = {}
            for what, c in items:
                n = lib.dgpu_encoder_item_bytes(self.enc.handle, pn, what, c)
                if n == 0:
                    continue
                b = self.bufs.get((what, c, n))
                if b is None:
                    b = self.bufs[(what, c, n)] = torch.empty(n, dtype=torch.uint8, pin_memory=True)
                rc = lib.dgpu_encoder_read(self.enc.handle, pn, what, c, b.data_ptr(), n, 1)
                if rc:
                    raise RuntimeError(f"dgpu_encoder_read failed: {rc}")
                self.d2h += n
                got[(what, c)] = b.numpy()
            return got

        def step_adaptive(self, src, loaded=False, outputs=None):
            """The stock encoder's choices (AdaptiveCoder): each picture's quantisers chosen with
            the entropy-correction factors of its kind adapted from the coded bytes of the
            pictures before it; a picture's bands are coded on a host thread while the pictures
            after it that do not depend on them are finished on the device."""
            if not loaded:
                self.load(src)
            infos, _, _ = self.coder.run_native(max_pictures=args.frames, keep_data=outputs is not None)
            self.pictures += len(infos)
            if outputs is not None:  # every picture keeps its slot: max_pictures = the sequence
                for info in infos:
                    outputs[info["pnum"]] = [self.enc.read(info["pnum"], E.OUTPUT, c) for c in range(3)]

        def load(self, src):
            enc = self.enc
            enc.reset()
            for f in src:
                enc.load(f)
            enc.end_sequence()

        def step(self, src, events=None, with_read=False, loaded=False):
            enc = self.enc
            if not loaded:
                self.load(src)
            infos = []
            while True:
                if events is not None:
                    e = torch.cuda.Event(enable_timing=True)
                    e.record(self.stream)
                    events.append(e)
                info = enc.code_next()
                if info is None:
                    return infos
                infos.append(info)
                if with_read:
                    self.read(info)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(ms):
        return max_over_ranks_ms(ms, world, "cuda")

    from concurrent.futures import ThreadPoolExecutor

    pools = {}

    def pool(key, n):
        """Host threads kept across timed runs (their page-locked staging buffers persist)."""
        if key not in pools:
            pools[key] = ThreadPoolExecutor(n)
        return pools[key]

    group_phases = {}  # host seconds per phase, summed over the groups of the last timed() run
    phase_lock = threading.Lock()

    def timed(lanes, src, steps, with_read=False, groups=None, adaptive=False):
        """Device time (ms) of `steps` sequence encodes on every lane, the lanes running
        concurrently: a start event on the main stream that every lane stream waits on, and an
        end event after the main stream has waited on every lane's last work.  With groups
        [(encoder group, its lanes)], each group's host thread repeats: load its lanes'
        sequences, run the group's batched motion estimation, code its lanes (a thread per
        lane); several groups run concurrently, so one group's estimation overlaps another's
        coding."""
        main = torch.cuda.current_stream()
        torch.cuda.synchronize()
        barrier()
        group_phases.clear()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(main)
        for ln in lanes:
            ln.stream.wait_event(e0)
            ln.d2h = 0
            ln.pictures = 0
            ln.coder.d2h_bytes = ln.coder.coded_bytes = 0

        def code(ln, loaded):
            if adaptive:
                ln.step_adaptive(src, loaded=loaded)
            else:
                ln.step(src, with_read=with_read, loaded=loaded)

        def run(ln):
            for _ in range(steps):
                code(ln, False)

        def add_phase(k, dt):
            with phase_lock:
                group_phases[k] = group_phases.get(k, 0.0) + dt

        def run_group(gi):
            slot = groups[gi]
            if len(slot) == 1:
                g, gl = slot[0]
                ex = pool(("group", gi, 0, len(gl)), len(gl))
                for _ in range(steps):
                    t0 = time.perf_counter()
                    list(ex.map(lambda ln: ln.load(src), gl))
                    t1 = time.perf_counter()
                    g.estimate()
                    t2 = time.perf_counter()
                    list(ex.map(lambda ln: code(ln, True), gl))
                    t3 = time.perf_counter()
                    for k, dt in (("load", t1 - t0), ("estimate", t2 - t1), ("code", t3 - t2)):
                        add_phase(k, dt)
                return
            # two sets alternate: step k runs on set k % 2; the estimation of step k + 1 (the
            # other set) runs while step k is coded, and a set is loaded again only after its
            # previous step's coding is done
            est_done = [threading.Event() for _ in range(steps)]
            code_done = [threading.Event() for _ in range(steps)]
            failed = []

            def estimator():
                try:
                    for k in range(steps):
                        g, gl = slot[k % 2]
                        if k >= 2:
                            code_done[k - 2].wait()
                            if failed:
                                return
                        ex = pool(("load", gi, k % 2, len(gl)), len(gl))
                        t0 = time.perf_counter()
                        list(ex.map(lambda ln: ln.load(src), gl))
                        t1 = time.perf_counter()
                        g.estimate()
                        add_phase("load", t1 - t0)
                        add_phase("estimate", time.perf_counter() - t1)
                        est_done[k].set()
                except BaseException as e:  # the coding thread must not wait for good
                    failed.append(e)
                    for ev in est_done:
                        ev.set()

            def coder():
                try:
                    for k in range(steps):
                        est_done[k].wait()
                        if failed:
                            return
                        g, gl = slot[k % 2]
                        ex = pool(("code", gi, k % 2, len(gl)), len(gl))
                        t0 = time.perf_counter()
                        list(ex.map(lambda ln: code(ln, True), gl))
                        add_phase("code", time.perf_counter() - t0)
                        code_done[k].set()
                except BaseException as e:
                    failed.append(e)
                    for ev in code_done:
                        ev.set()

            th = [threading.Thread(target=estimator), threading.Thread(target=coder)]
            for t in th:
                t.start()
            for t in th:
                t.join()
            if failed:
                raise failed[0]

        if groups is not None:
            list(pool(("groups", len(groups)), len(groups)).map(run_group, range(len(groups))))
        elif len(lanes) == 1:
            run(lanes[0])
        else:
            list(pool(("lanes", len(lanes)), len(lanes)).map(run, lanes))
        for ln in lanes:
            done = torch.cuda.Event()
            done.record(ln.stream)
            main.wait_event(done)
        e1.record(main)
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1))

    if lib.dgpu_me_set_occupancy(args.me_occupancy):
        raise ValueError("--me-occupancy must be 1..8")
    if lib.dgpu_me_set_unit_lifetime(args.me_unit_life):
        raise ValueError("--me-unit-life must be >= 0")
    if lib.dgpu_set_blocking_waits(args.blocking_waits):
        raise ValueError("--blocking-waits must be 0 or 1")
    nsets = 2 if args.double_buffer else 1
    lanes = [Lane() for _ in range(args.streams * nsets)]
    sets = [lanes[i * args.streams:(i + 1) * args.streams] for i in range(nsets)]
    lanes_a = sets[0]  # the forms that run one set of sequences
    plain = lanes[0]
    # the batched form: the lanes split into --me-groups encoder groups that run concurrently
    ng = max(1, min(args.me_groups, args.streams))
    per = (args.streams + ng - 1) // ng
    groups = [[(E.EncoderGroup([ln.enc for ln in st[k:k + per]]), st[k:k + per]) for st in sets]
              for k in range(0, args.streams, per)]

    # ---- warm-up: every lane, both input forms ------------------------------------------------
    for _ in range(args.warmup):
        timed(lanes, dev_frames, nsets, groups=groups)  # every set
    timed(lanes, pinned_np, nsets, groups=groups, adaptive=True)

    # ---- the integer roofline and the motion-estimation kernels' algorithmic operations -------
    rate = ctypes.c_double(0.0)
    if lib.dgpu_measure_int_rate(ctypes.byref(rate)):
        raise RuntimeError("dgpu_measure_int_rate failed")
    int_peak = rate.value / 1e9  # Gop/s
    ops_dev = torch.zeros(3, dtype=torch.int64, device="cuda")
    lib.dgpu_debug_wavefront(-1, 0, None, None, None, ops_dev.data_ptr())
    lib.dgpu_me_profile(1, None, None)
    timed(lanes, dev_frames, 1, groups=groups)  # one batched step, counted (untimed)
    count_launches = (ctypes.c_int * 7)()
    lib.dgpu_me_profile(0, None, count_launches)
    lib.dgpu_debug_wavefront(-1, 0, None, None, None, None)
    me_ops_per_step = [int(x) for x in ops_dev.cpu().tolist()]

    # ---- timed region (batched form): inputs resident in HBM ---------------------------------
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    launches0 = lib.dgpu_launch_count()
    lib.dgpu_me_profile(1, None, None)  # CUDA events around each motion-estimation kernel
    ms = timed(lanes, dev_frames, args.steps, groups=groups)
    me_ms = (ctypes.c_double * 7)()
    me_launches = (ctypes.c_int * 7)()
    lib.dgpu_me_profile(0, me_ms, me_launches)
    launches = lib.dgpu_launch_count() - launches0
    clk = clocks.stop()
    frames_per_step = args.frames * args.streams  # one set of sequences per step
    ms_per_step = ms / args.steps
    value = whole_job_rate(world, frames_per_step, args.steps, ms)

    # ---- end to end (batched form) through the C ABI with host buffers, stock choices ---------
    # pinned host frames in; per picture the quantised indices, band and code-block choices
    # and motion data out; every picture's subbands arithmetic-coded on the host and the
    # entropy-correction state adapted from the byte counts, so the quantiser choices are the
    # stock reference encoder's
    ru0, w0 = resource.getrusage(resource.RUSAGE_SELF), time.perf_counter()
    ems = timed(lanes, pinned_np, args.steps, groups=groups, adaptive=True)
    ru1, w1 = resource.getrusage(resource.RUSAGE_SELF), time.perf_counter()
    cpu_s = (ru1.ru_utime - ru0.ru_utime) + (ru1.ru_stime - ru0.ru_stime)
    h2d = sum(p.nbytes for fr in pinned_np for p in fr) * args.streams
    e2e = {"value": whole_job_rate(world, frames_per_step, args.steps, ems), "unit": "frames/s",
           "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": sum(ln.d2h + ln.coder.d2h_bytes for ln in lanes) // args.steps,
           "coded_band_bytes_per_step": sum(ln.coder.coded_bytes for ln in lanes) // args.steps,
           "form": "stock choices: adaptive entropy-correction factors, subbands arithmetic-coded on the host",
           "pipeline": "dgpu_encoder_code_adaptive: a picture waits only for the host coding of the last "
                       "picture of its kind (intra, B, other inter), whose factors it reads; inter pictures' "
                       "indices copied as int16 when their coefficients fit",
           "group_ms_per_step": {k: round(1000.0 * v / (args.steps * len(groups)), 2) for k, v in group_phases.items()},
           "host_cpu": {"cores_busy": round(cpu_s / (w1 - w0), 2), "cores": os.cpu_count(),
                        "ms_per_picture": round(1000.0 * cpu_s / (frames_per_step * args.steps), 3)}}
    # the same without host coding (initial factors kept): the hot path alone through the ABI
    hms = timed(lanes, pinned_np, args.steps, with_read=True, groups=groups)
    e2e_hot = {"value": whole_job_rate(world, frames_per_step, args.steps, hms), "unit": "frames/s",
               "form": "initial entropy-correction factors, no host coding"}

    # ---- batched form without the group: concurrent sequences, each estimating alone -----------
    sms = timed(lanes_a, dev_frames, args.steps)
    streams_only = {"value": whole_job_rate(world, frames_per_step, args.steps, sms), "unit": "frames/s",
                    "ms_per_step": sms / args.steps,
                    "form": f"{len(lanes_a)} concurrent sequences, each with its own motion-estimation launches"}
    g_all = E.EncoderGroup([ln.enc for ln in lanes_a])
    oms = timed(lanes_a, dev_frames, args.steps, groups=[[(g_all, lanes_a)]])
    g_all.close()
    one_group = {"value": whole_job_rate(world, frames_per_step, args.steps, oms), "unit": "frames/s",
                 "ms_per_step": oms / args.steps,
                 "form": f"{len(lanes_a)} sequences in one encoder group (estimation, then coding)"}

    # ---- plain form: one sequence at a time ----------------------------------------------------
    pms = timed([plain], dev_frames, args.steps)
    pems = timed([plain], pinned_np, args.steps, adaptive=True)
    plain_line = {"value": world * args.frames * args.steps / (pms / 1000.0), "ms_per_step": pms / args.steps,
                  "e2e": world * args.frames * args.steps / (pems / 1000.0), "unit": "frames/s",
                  "batched_over_plain": value / (world * args.frames * args.steps / (pms / 1000.0))}

    # ---- self-check: the timed sequence coded with the stock choices equals the reference's ----
    parity = None
    if ref_recon is not None:
        outs = {}
        plain.step_adaptive(pinned_np, outputs=outs)
        same = len(outs) == args.frames and all(
            np.array_equal(outs[i][c], np.ascontiguousarray(ref_recon[i][c]).ravel())
            for i in range(args.frames) for c in range(3))
        parity = {"frames": args.frames, "locally_decoded_equal_reference": bool(same),
                  "form": "the step's whole sequence coded as the e2e form codes it (stock adaptive factors, host "
                          "band coding), every locally decoded plane compared with the reference encoder's own "
                          "(its cpu_baseline run)"}

    # ---- per-picture latency of the plain form (device timeline, coding order) ---------------
    lat = []
    for _ in range(max(1, args.steps)):
        evs = []
        plain.step(dev_frames, events=evs)
        plain.stream.synchronize()
        lat += [evs[k].elapsed_time(evs[k + 1]) for k in range(len(evs) - 1)]
    lat.sort()
    latency = {"p50": statistics.median(lat), "p99": lat[min(len(lat) - 1, int(round(0.99 * (len(lat) - 1))))],
               "max": lat[-1], "pictures": len(lat), "form": "plain"}

    # ---- stage breakdown (plain form): the streaming kernels against the HBM roofline ---------
    enc = plain.enc
    enc.profile(True)
    reps = 2
    for _ in range(reps):
        infos = plain.step(dev_frames)
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
    peak_source = ("MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks
                   else "fallback 6650 GB/s (of fallback)")
    streaming = {}
    for k, kern in STREAMING_KERNELS.items():
        if stage_ms.get(k, 0.0) <= 0:
            continue
        gbs = alg[k] / (stage_ms[k] / 1000.0) / 1e9
        streaming[k] = {"kernels": kern, "ms_per_sequence": round(stage_ms[k], 3), "algorithmic_bytes": alg[k],
                        "gbs": round(gbs, 1), "frac": round(gbs / peak, 4)}

    # ---- the motion-estimation kernels against the integer roofline (batched timed region) ----
    def me_kernel(name, key):
        t = sum(me_ms[c] for c in ME_CLASSES[key])
        n = sum(me_launches[c] for c in ME_CLASSES[key])
        ops = me_ops_per_step[ME_OP_INDEX[key]] * args.steps
        achieved = ops / (t / 1000.0) / 1e9 if t > 0 else 0.0
        return {"kernels": name, "ms_total": round(t, 3), "launches": n, "algorithmic_ops": ops,
                "achieved": round(achieved, 1), "frac": round(achieved / int_peak, 4)}

    me_kernels = {"pel_search": me_kernel("pel_lists_kernel + pel_wavefront_kernel", "pel_search"),
                  "subpel_refinement": me_kernel("subpel_wavefront_kernel", "subpel_refinement"),
                  "mode_decision": me_kernel("mode_blocks_kernel + mode_wavefront_kernel", "mode_decision")}
    dom = max(me_kernels, key=lambda k: me_kernels[k]["ms_total"])
    d = me_kernels[dom]
    per_launch_ops = me_ops_per_step[ME_OP_INDEX[dom]] / max(1, sum(count_launches[c] for c in ME_CLASSES[dom]))
    traffic = ME_TRAFFIC_PER_OP.get(dom)
    roofline = {"bound": "int", "kernel": d["kernels"], "achieved": d["achieved"], "peak": round(int_peak, 1),
                "unit": "Gop/s", "frac": d["frac"],
                "traffic": round(traffic * per_launch_ops) if traffic else None,
                "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of the 13-frame "
                                  "encode leg (profiles/encoder_1080p13_dram_traffic.md), scaled to this launch by "
                                  "its algorithmic operations" if traffic else None,
                "peak_source": "dgpu_measure_int_rate: acc += |a - b| on every SM, 3 operations per term "
                               "(measured in this run)",
                "algorithmic_ops": "3 per pixel of every block difference the reference's search evaluates, plus "
                                   "sub-pel interpolation (4 per pixel at quarter-pel), bi-prediction and intra terms "
                                   "(counted on the device in an untimed step)",
                "ops_per_launch": round(per_launch_ops),
                "me_kernels": me_kernels, "streaming_kernels": streaming,
                "streaming_peak": {"value": peak, "unit": "GB/s", "source": peak_source},
                "note": "motion-estimation kernel times: CUDA events around each launch on the encoder groups' "
                        "streams inside the timed region (concurrent groups' times add up); streaming kernels: "
                        "plain form, encoder stage events in a separate pass"}
    # ---- decoding: the plain form's coded sequence through the device decoder ----------------
    decoding = None
    if args.decode and world == 1:
        decoding = run_decoding(args, enc, infos, peak, cpu_decode)
    for slot in groups:
        for g, _ in slot:
            g.close()
    for ln in lanes:
        ln.enc.close()
    for ex in pools.values():
        ex.shutdown()

    # ---- heterogeneous picture batch: 64 mixed pictures coded together (one GPU) ----------------
    hetero = None
    if args.hetero_steps > 0:
        hetero = run_hetero(args, peak, peaks)

    # ---- serving loop: Poisson arrivals of live streams of mixed sizes (one GPU) ----------------
    serving = None
    if args.serving_seconds > 0 and world == 1:
        from dirac_b200 import serving as S

        cfg = {"seconds": args.serving_seconds, "arrivals_per_s": args.serving_rate, "fps_per_stream": 50,
               "resolutions": "352x288, 720x576, 1280x720, 1920x1080, 3840x2160 (4:2:0, 8- or 10-bit)",
               "frames_per_stream": "8-64", "budget_gb": 80, "max_active": 40, "max_load": 16,
               "input": "per resolution and depth a pool of synthetic frames (16; 8 at 3840x2160), each stream "
                        "cycling through its pool from a random offset"}
        try:
            reqs = S.make_requests(args.serving_seconds, args.serving_rate, ["cif", "576", "720", "1080", "2160"], 8, 64,
                                   seed=7,
                                   depths=(8, 10))
            serving = S.ServingLoop(int(80e9), max_active=40, frame_interval=1.0 / 50, batch_me=True,
                                    max_load=16).run(reqs)
        except Exception as e:  # the serving leg must not cost the bench line; its failure is reported
            serving = {"error": repr(e)}
        serving["config"] = cfg

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
                "config": {"workload": workload_name(args.frames), "frames_per_step": frames_per_step,
                           "global_batch": world * frames_per_step, "parallelism": f"replicas{world}",
                           "form": f"batched: {args.streams} sequences per step in {len(groups)} encoder groups "
                                   "running concurrently; each group's motion estimation in one batched launch, "
                                   "each sequence's coding on its own stream and host thread"
                                   + ("; each group alternates two sets of sequences, one set's estimation "
                                      "running while the other set is coded" if nsets == 2 else ""),
                           "me_ctas_per_sm": args.me_occupancy, "me_unit_life": args.me_unit_life,
                           "lane_priority": args.lane_priority, "blocking_waits": args.blocking_waits,
                           "l2": "inputs and working set larger than L2 (no flush needed)"},
                "e2e": e2e, "cpu_baseline": cpu_baseline, "parity_vs_reference": parity, "plain": plain_line,
                "gpu_launches": launches, "clocks": clk, "e2e_hot_path": e2e_hot, "roofline": roofline,
                "batched_one_group": one_group, "batched_streams_only": streams_only, "latency_ms": latency,
                "heterogeneous_batch": hetero, "serving": serving, "decoding": decoding}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
