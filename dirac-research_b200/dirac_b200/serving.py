"""Serving loop: encode streams as they arrive, admitted against a device-memory budget.

Each request is a sequence of frames of its own size and bit depth.  A request is admitted as
soon as its encoder's device memory (``encoder.device_bytes``) fits in what the budget has
left; until then it waits in arrival order.  Every admitted stream gets its own encoder, CUDA
stream and host thread, so work from streams that arrive while others are on the GPU overlaps
on the device (continuous admission, not a queue of whole jobs).  With batch_me, the streams of
one picture format also share their motion estimation: a stream that has loaded a frame joins
its format's MeBatcher, and one launch (dgpu_encoders_estimate) estimates the estimable
pictures of every stream that joined within a short window.  Frames of a stream become
available one frame interval apart from its arrival (live encoding); a picture's latency is
the time from its frame's availability to the end of its coding on the device, reported apart
from the admission wait (arrival to admission).  Results of a stream do not depend on what
runs beside it: the encoders share no state, and an estimate is the same in any batch.

    python -m dirac_b200.serving --seconds 10 --rate 4 --budget-gb 40
"""
import argparse
import json
import statistics
import threading
import time

from . import _lib


class Request:
    """One stream: params (encoder parameter dict), frames (host sample planes per frame),
    arrival (seconds after the loop starts), optional name."""

    def __init__(self, params, frames, arrival=0.0, name=None):
        self.params = params
        self.frames = frames
        self.arrival = arrival
        self.name = name


class MeBatcher:
    """Motion estimation shared by the live streams of one picture format.  A stream thread that
    has loaded new frames calls estimate(encoder) and blocks.  One waiting thread at a time leads:
    it waits `window` seconds for other streams to join, then estimates the oldest joined
    encoders' estimable pictures in one dgpu_encoders_estimate launch (their threads are all
    waiting, so no encoder is in use elsewhere) and releases them, round after round until its
    own encoder is done; then the lead passes to a waiting thread.  A round holds at most
    max_batch encoders and at most ws_limit bytes of workspace (always at least one encoder);
    the workspace grows to the largest round.  An error fails only the round it happened in."""

    def __init__(self, window=0.002, max_batch=8, ws_limit=2 << 30):
        self.lib = None        # library and stream made by the first round
        self.stream = None
        self.window = window
        self.max_batch = max_batch
        self.ws_limit = ws_limit
        self.cv = threading.Condition()
        self.pending = []      # entries {"enc", "done", "error"} in arrival order
        self.leading = False
        self.ws = None
        self.rounds = 0
        self.batched = 0       # encoders estimated, summed over rounds
        self.tasks = 0

    def estimate(self, enc):
        entry = {"enc": enc, "done": False, "error": None}
        with self.cv:
            self.pending.append(entry)
            while not entry["done"] and self.leading:
                self.cv.wait()
            lead = not entry["done"]
            if lead:
                self.leading = True
        if lead:
            try:
                while not entry["done"]:
                    time.sleep(self.window)
                    with self.cv:
                        batch = self._take()
                    try:
                        self._run([e["enc"] for e in batch])
                    except Exception as ex:  # reported to every member of this round
                        for e in batch:
                            e["error"] = repr(ex)
                    with self.cv:
                        for e in batch:
                            e["done"] = True
                        self.cv.notify_all()
            finally:
                with self.cv:
                    if not entry["done"] and entry in self.pending:
                        self.pending.remove(entry)
                    self.leading = False
                    self.cv.notify_all()
        if entry["error"]:
            raise RuntimeError(entry["error"])

    def _load(self):
        if self.lib is None:
            from . import _lib

            self.lib = _lib.load()
        return self.lib

    def _need(self, encs):
        from . import _lib

        return self._load().dgpu_encoder_group_device_bytes(_lib.ptr_array([e.handle.value for e in encs]), len(encs))

    def _take(self):
        """The oldest pending entries that fit max_batch and ws_limit (at least one); removed from
        the pending list.  Called with the lock held."""
        n = min(len(self.pending), self.max_batch)
        while n > 1 and self._need([e["enc"] for e in self.pending[:n]]) > self.ws_limit:
            n -= 1
        batch = self.pending[:n]
        del self.pending[:n]
        return batch

    def _run(self, encs):
        import ctypes

        import torch

        from . import _lib

        if self.stream is None:
            self.stream = torch.cuda.Stream()
        handles = _lib.ptr_array([e.handle.value for e in encs])
        need = self._load().dgpu_encoder_group_device_bytes(handles, len(encs))
        if need == 0:
            raise ValueError("encoders of different formats in one estimation")
        if self.ws is None or self.ws.numel() < need:
            self.ws = None
            self.ws = torch.empty(need, dtype=torch.uint8, device="cuda")
        n = ctypes.c_int(0)
        _lib.check(self.lib.dgpu_encoders_estimate(handles, len(encs), self.ws.data_ptr(), self.ws.numel(),
                                                   self.stream.cuda_stream, ctypes.byref(n)), "dgpu_encoders_estimate")
        self.rounds += 1
        self.batched += len(encs)
        self.tasks += n.value


class ServingLoop:
    def __init__(self, budget_bytes, max_active=16, frame_interval=0.0, slots=24, collect=None,
                 encoder_factory=None, bytes_fn=None, batch_me=False, max_load=16):
        """budget_bytes: device memory the loop may give to encoders.  max_active: streams
        coded at once.  frame_interval: seconds between a stream's frames (0: all at arrival).
        slots: picture slots per encoder.  collect(request, encoder, info): called after each
        coded picture (e.g. to read results).  encoder_factory / bytes_fn: injectable for tests.
        batch_me: share motion-estimation launches between the live streams of one format.
        max_load: frames a stream loads at most before each estimation round (all that are due,
        when it runs behind)."""
        self.budget = budget_bytes
        self.max_active = max_active
        self.frame_interval = frame_interval
        self.slots = slots
        self.collect = collect
        self.batch_me = batch_me
        self.max_load = max(1, max_load)
        self.batchers = {}
        self.warm = encoder_factory is None
        if encoder_factory is None:
            from .encoder import SequenceEncoder

            def encoder_factory(params, max_pictures):
                import torch

                return SequenceEncoder(params, max_pictures=max_pictures, stream=torch.cuda.Stream())
        if bytes_fn is None:
            from .encoder import device_bytes as bytes_fn
        self.encoder_factory = encoder_factory
        self.bytes_fn = bytes_fn

    def _slots_for(self, req):
        return min(len(req.frames), self.slots)

    def run(self, requests):
        """Serve every request; returns a dict of statistics (latencies in ms)."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        for r in reqs:
            r.need = self.bytes_fn(r.params, self._slots_for(r))
            if r.need > self.budget:
                raise ValueError(f"request {r.name} needs {r.need} bytes, more than the whole budget")
        if self.warm:
            # CUDA context, library and kernel modules initialised before the clock starts
            # (the first initialisation holds the interpreter lock for a while)
            self.encoder_factory(params_for(64, 64), 1).close()
        lock = threading.Condition()
        state = {"free": self.budget, "active": 0, "peak_active": 0, "peak_bytes": 0, "errors": []}
        lat = []
        frames_done = [0]
        t0 = time.perf_counter()

        def batcher_for(r):
            if not self.batch_me:
                return None
            key = tuple(sorted(r.params.items()))
            with lock:
                if key not in self.batchers:
                    self.batchers[key] = MeBatcher()
                return self.batchers[key]

        def worker(r):
            try:
                enc = self.encoder_factory(r.params, self._slots_for(r))
                batcher = batcher_for(r)
                avail = {}
                pending = []

                def drain():
                    while True:
                        info = enc.code_next()
                        if info is None:
                            return
                        pending.append(info)
                        if hasattr(enc, "stream"):
                            enc.stream.synchronize()
                        now = time.perf_counter()
                        with lock:
                            lat.append(1000.0 * (now - avail[info["pnum"]]))
                            frames_done[0] += 1
                        if self.collect is not None:
                            self.collect(r, enc, info)

                i, nfr = 0, len(r.frames)
                while i < nfr:
                    due = t0 + r.arrival + i * self.frame_interval
                    wait = due - time.perf_counter()
                    if wait > 0:
                        time.sleep(wait)
                    # every frame already due (a stream admitted late has many) goes in before
                    # one estimation round, up to max_load and while the encoder has free slots
                    now = time.perf_counter()
                    k = 0
                    while i < nfr and k < self.max_load and (k == 0 or t0 + r.arrival + i * self.frame_interval <= now):
                        try:
                            enc.load(r.frames[i])
                        except _lib.DgpuError as e:
                            if e.code != _lib.DGPU_ERR_SIZE or k == 0:
                                raise
                            break  # no free slot: code what is loaded first
                        avail[i] = max(t0 + r.arrival + i * self.frame_interval, t0 + r.arrival)
                        i += 1
                        k += 1
                    if batcher is not None:
                        batcher.estimate(enc)
                    drain()
                enc.end_sequence()
                if batcher is not None:
                    batcher.estimate(enc)
                drain()
                enc.close()
            except Exception as e:  # reported after the loop, never swallowed
                with lock:
                    state["errors"].append(f"{r.name}: {e!r}")
            finally:
                with lock:
                    state["free"] += r.need
                    state["active"] -= 1
                    lock.notify_all()

        threads = []
        queue = list(reqs)
        waits = []
        with lock:
            while queue:
                r = queue[0]
                now = time.perf_counter() - t0
                if now < r.arrival:
                    lock.wait(timeout=r.arrival - now)
                    continue
                if r.need > state["free"] or state["active"] >= self.max_active:
                    lock.wait(timeout=0.05)
                    continue
                queue.pop(0)
                waits.append(1000.0 * (time.perf_counter() - t0 - r.arrival))
                state["free"] -= r.need
                state["active"] += 1
                state["peak_active"] = max(state["peak_active"], state["active"])
                state["peak_bytes"] = max(state["peak_bytes"], self.budget - state["free"])
                th = threading.Thread(target=worker, args=(r,), daemon=True)
                th.start()
                threads.append(th)
        for th in threads:
            th.join()
        wall = time.perf_counter() - t0
        if state["errors"]:
            raise RuntimeError("; ".join(state["errors"]))
        lat.sort()

        def pct(p):
            return lat[min(len(lat) - 1, int(round(p * (len(lat) - 1))))] if lat else None

        return {"streams": len(reqs), "pictures": frames_done[0], "wall_s": wall,
                "frames_per_s": frames_done[0] / wall if wall > 0 else None,
                "latency_ms": {"p50": pct(0.5), "p99": pct(0.99), "max": lat[-1] if lat else None},
                "admission_wait_ms": {"p50": statistics.median(waits) if waits else None,
                                      "p99": sorted(waits)[min(len(waits) - 1, int(round(0.99 * (len(waits) - 1))))]
                                      if waits else None,
                                      "max": max(waits) if waits else None},
                "peak_active": state["peak_active"], "peak_bytes": state["peak_bytes"],
                "budget_bytes": self.budget,
                "shared_estimation": {"rounds": sum(b.rounds for b in self.batchers.values()),
                                      "streams_per_round": (sum(b.batched for b in self.batchers.values()) /
                                                            max(1, sum(b.rounds for b in self.batchers.values()))),
                                      "estimates": sum(b.tasks for b in self.batchers.values())}
                if self.batch_me else None}


RESOLUTIONS = {"cif": (352, 288), "576": (720, 576), "720": (1280, 720), "1080": (1920, 1080),
               "2160": (3840, 2160)}


def params_for(w, h, depth=8):
    """Coding parameters of a served stream (4:2:0, the bench's GOP, QF and block sizes)."""
    return dict(cformat=2, width=w, height=h, luma_depth=depth, chroma_depth=depth, qf=7.0, l1_sep=3, num_l1=7,
                cpd=32.0, xblen=16, yblen=16, xbsep=12, ybsep=12, mv_precision=2, intra_filter=6, inter_filter=0,
                wlt_depth=4)


def make_requests(seconds, rate, resolutions, min_frames, max_frames, seed=0, pool_frames=16, depths=(8,)):
    """Poisson arrivals at `rate` streams/s over `seconds`; each stream a resolution drawn
    uniformly from `resolutions` and a bit depth from `depths`, a length uniform in
    [min_frames, max_frames], and frames taken (cycled from a per-stream offset) from a seeded
    synthetic pool per resolution and depth (pool_frames frames; half as many for 3840x2160,
    whose generation on the host is slow)."""
    import numpy as np

    from . import synth

    rng = np.random.default_rng(seed)
    pools = {}
    reqs = []
    t = 0.0
    k = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            break
        res = resolutions[rng.integers(len(resolutions))]
        depth = int(depths[rng.integers(len(depths))])
        w, h = RESOLUTIONS[res]
        npool = max(2, pool_frames // 2) if w * h > 1920 * 1088 else pool_frames
        if (res, depth) not in pools:
            pools[(res, depth)] = synth.make_sequence(w, h, npool, n_rects=8, vmax=8, seed=100 + len(pools),
                                                      bit_depth=depth)
        pool = pools[(res, depth)]
        n = int(rng.integers(min_frames, max_frames + 1))
        off = int(rng.integers(npool))
        frames = [pool[(off + i) % npool] for i in range(n)]
        reqs.append(Request(params_for(w, h, depth), frames, t, f"s{k}-{res}-{depth}bit-x{n}"))
        k += 1
    return reqs


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--seconds", type=float, default=10.0)
    ap.add_argument("--rate", type=float, default=4.0, help="stream arrivals per second (Poisson)")
    ap.add_argument("--budget-gb", type=float, default=40.0)
    ap.add_argument("--max-active", type=int, default=16)
    ap.add_argument("--fps", type=float, default=50.0, help="frame rate of the live streams (0: all at once)")
    ap.add_argument("--resolutions", default="cif,576,720,1080")
    ap.add_argument("--frames", default="8-64")
    ap.add_argument("--depths", default="8", help="bit depths drawn per stream, e.g. 8,10")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--batch-me", type=int, default=1, help="1: streams of one format share estimation launches")
    ap.add_argument("--max-load", type=int, default=16, help="frames a stream loads at most per estimation round")
    a = ap.parse_args(argv)
    lo, hi = (int(x) for x in a.frames.split("-"))
    reqs = make_requests(a.seconds, a.rate, a.resolutions.split(","), lo, hi, a.seed,
                         depths=[int(d) for d in a.depths.split(",")])
    loop = ServingLoop(int(a.budget_gb * 1e9), a.max_active, 1.0 / a.fps if a.fps > 0 else 0.0,
                       batch_me=bool(a.batch_me), max_load=a.max_load)
    stats = loop.run(reqs)
    stats["config"] = {"seconds": a.seconds, "rate": a.rate, "resolutions": a.resolutions, "frames": a.frames,
                       "depths": a.depths, "fps": a.fps, "budget_gb": a.budget_gb, "batch_me": bool(a.batch_me),
                       "max_active": a.max_active, "max_load": a.max_load}
    print(json.dumps(stats))
    return 0


if __name__ == "__main__":
    import sys

    sys.exit(main())
