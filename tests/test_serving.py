"""Serving loop: admission against the device-memory budget, continuous admission of
arriving streams, latency accounting (CPU, with a stand-in encoder), and on the GPU the
identity of every stream's results alone and in the mix."""
import threading
import time

import numpy as np
import pytest


class FakeEncoder:
    """Codes each loaded picture at the next code_next call after a short pause, tracking
    how many bytes are live across all fakes."""

    live = 0
    peak = 0
    lock = threading.Lock()

    def __init__(self, params, max_pictures):
        self.need = params["bytes"]
        with FakeEncoder.lock:
            FakeEncoder.live += self.need
            FakeEncoder.peak = max(FakeEncoder.peak, FakeEncoder.live)
        self.loaded = []
        self.next = 0
        self.done = False

    def load(self, frame):
        self.loaded.append(frame)

    def end_sequence(self):
        self.done = True

    def code_next(self):
        if self.next < len(self.loaded):
            time.sleep(0.002)
            self.next += 1
            return {"pnum": self.next - 1}
        return None

    def close(self):
        with FakeEncoder.lock:
            FakeEncoder.live -= self.need


def test_admission_respects_budget_and_serves_everything():
    from dirac_b200.serving import Request, ServingLoop

    FakeEncoder.live = FakeEncoder.peak = 0
    reqs = [Request({"bytes": 300 + 100 * (k % 3)}, list(range(5 + k % 4)), arrival=0.01 * k, name=str(k))
            for k in range(12)]
    coded = {}

    def collect(r, enc, info):
        coded.setdefault(r.name, []).append(info["pnum"])

    loop = ServingLoop(budget_bytes=1000, max_active=8, frame_interval=0.001, collect=collect,
                       encoder_factory=FakeEncoder, bytes_fn=lambda p, n: p["bytes"])
    stats = loop.run(reqs)
    assert FakeEncoder.peak <= 1000 and FakeEncoder.live == 0
    assert stats["peak_bytes"] <= 1000 and stats["peak_active"] >= 2
    assert stats["pictures"] == sum(len(r.frames) for r in reqs)
    for r in reqs:
        assert coded[r.name] == list(range(len(r.frames)))
    assert stats["latency_ms"]["p50"] > 0 and stats["latency_ms"]["p99"] >= stats["latency_ms"]["p50"]


def test_frames_already_due_load_together_within_free_slots():
    """A stream whose frames are all due when it starts loads several of them before each
    coding pass (one estimation round for many pictures), stops at a refused load (no free
    slot: DGPU_ERR_SIZE) and codes first; every picture is coded, in order."""
    from dirac_b200 import _lib
    from dirac_b200.serving import Request, ServingLoop

    log = []

    class SlotEncoder(FakeEncoder):
        def load(self, frame):
            if len(self.loaded) - self.next >= 3:
                raise _lib.DgpuError(_lib.DGPU_ERR_SIZE, "dgpu_encoder_load")
            log.append("L")
            super().load(frame)

        def code_next(self):
            info = super().code_next()
            if info is not None:
                log.append("C")
            return info

    FakeEncoder.live = FakeEncoder.peak = 0
    coded = []
    loop = ServingLoop(budget_bytes=1000, max_active=1, frame_interval=0.0, encoder_factory=SlotEncoder,
                       bytes_fn=lambda p, n: p["bytes"], collect=lambda r, e, i: coded.append(i["pnum"]))
    loop.run([Request({"bytes": 100}, list(range(10)), name="late")])
    assert coded == list(range(10))
    runs = "".join(log).split("C")
    assert max(len(x) for x in runs) == 3 and log.count("L") == 10


def test_request_larger_than_budget_is_refused():
    from dirac_b200.serving import Request, ServingLoop

    loop = ServingLoop(budget_bytes=100, encoder_factory=FakeEncoder, bytes_fn=lambda p, n: p["bytes"])
    with pytest.raises(ValueError):
        loop.run([Request({"bytes": 200}, [0, 1])])


def _batcher_class():
    from dirac_b200.serving import MeBatcher

    class FakeBatcher(MeBatcher):
        """Rounds recorded instead of launched; 100 bytes of workspace per encoder; a round that
        holds `fail_on` fails."""

        def __init__(self, fail_on=None, **kw):
            super().__init__(**kw)
            self.runs = []
            self.fail_on = fail_on

        def _need(self, encs):
            return 100 * len(encs)

        def _run(self, encs):
            self.runs.append(list(encs))
            time.sleep(0.001)
            if self.fail_on in encs:
                raise RuntimeError("estimation failed")

    return FakeBatcher


def _drive(batcher, nthreads, calls):
    errors = [0] * nthreads

    def worker(k):
        for _ in range(calls):
            try:
                batcher.estimate(k)
            except RuntimeError:
                errors[k] += 1
            time.sleep(0.0005 * (k % 3))

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(nthreads)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=60)
    assert not any(t.is_alive() for t in threads), "a stream stayed blocked in estimate"
    return errors


def test_shared_estimation_rounds_cover_every_call_once():
    """Every estimate call is served by exactly one round; no round holds an encoder twice or
    more than max_batch encoders or ws_limit bytes; rounds do batch several streams."""
    batcher = _batcher_class()(window=0.002, max_batch=4, ws_limit=300)
    errors = _drive(batcher, 12, 6)
    assert errors == [0] * 12
    counts = {}
    for r in batcher.runs:
        assert len(r) == len(set(r)) and 1 <= len(r) <= 3, r
        for k in r:
            counts[k] = counts.get(k, 0) + 1
    assert counts == {k: 6 for k in range(12)}
    assert max(len(r) for r in batcher.runs) > 1
    assert not batcher.pending and not batcher.leading


def test_shared_estimation_error_fails_only_its_round():
    """A failing round raises in the threads whose encoders it held, and only there; later
    rounds run normally."""
    batcher = _batcher_class()(fail_on=3, window=0.002, max_batch=4)
    errors = _drive(batcher, 8, 5)
    failed = [r for r in batcher.runs if 3 in r]
    assert errors[3] == 5 and len(failed) == 5
    for k in range(8):
        assert errors[k] == sum(k in r for r in failed), (k, errors)
    assert sum(len(r) for r in batcher.runs) == 40


def test_shared_estimation_round_of_one_above_the_workspace_limit():
    """An encoder whose workspace alone exceeds ws_limit is still estimated, in a round of one."""
    batcher = _batcher_class()(window=0.001, max_batch=8, ws_limit=50)
    assert _drive(batcher, 4, 3) == [0] * 4
    assert all(len(r) == 1 for r in batcher.runs) and len(batcher.runs) == 12


def test_encoder_device_bytes_grows_with_size_and_slots():
    from dirac_b200 import encoder as E
    from dirac_b200.serving import params_for

    a = E.device_bytes(params_for(352, 288), 16)
    b = E.device_bytes(params_for(1920, 1080), 16)
    c = E.device_bytes(params_for(1920, 1080), 40)
    assert 0 < a < b < c


@pytest.mark.gpu
@pytest.mark.parametrize("batch_me", [False, True], ids=["own", "shared"])
def test_served_streams_equal_alone_and_in_the_mix(gpu, batch_me):
    """Three streams of different sizes coded one at a time and then concurrently (admitted
    together, overlapping on the device; with shared estimation rounds per format): every
    picture's output samples and quantised indices are identical."""
    from dirac_b200 import synth
    from dirac_b200.encoder import OUTPUT, QINDEX
    from dirac_b200.serving import Request, ServingLoop, params_for

    specs = [(176, 144, 9, 1), (352, 288, 8, 2), (320, 240, 10, 3)]
    reqs = [Request(params_for(w, h), synth.make_sequence(w, h, n, n_rects=4, vmax=6, seed=s), 0.0, f"r{s}")
            for w, h, n, s in specs]

    def run(max_active):
        out = {}
        lock = threading.Lock()

        def collect(r, enc, info):
            pn = info["pnum"]
            got = [enc.read(pn, OUTPUT, c) for c in range(3)] + [enc.read(pn, QINDEX, c) for c in range(3)]
            with lock:
                out[(r.name, pn)] = got

        ServingLoop(budget_bytes=int(8e9), max_active=max_active, collect=collect, batch_me=batch_me).run(reqs)
        return out

    alone = run(1)
    mixed = run(3)
    assert alone.keys() == mixed.keys() and len(alone) == sum(n for _, _, n, _ in specs)
    for k in alone:
        for a, b in zip(alone[k], mixed[k]):
            np.testing.assert_array_equal(a, b, err_msg=str(k))


@pytest.mark.gpu
def test_shared_estimation_rounds_give_each_stream_its_own_results(gpu):
    """Four live streams of one format whose motion estimation runs in shared launches
    (MeBatcher, dgpu_encoders_estimate): every picture equals the same stream coded alone with
    its encoder's own estimation, and the rounds did batch several streams."""
    from dirac_b200 import synth
    from dirac_b200.encoder import MV, OUTPUT, QINDEX
    from dirac_b200.serving import Request, ServingLoop, params_for

    reqs = [Request(params_for(176, 144), synth.make_sequence(176, 144, 10, n_rects=4, vmax=6, seed=40 + k),
                    0.0, f"q{k}") for k in range(4)]

    def run(max_active, batch_me):
        out = {}
        lock = threading.Lock()

        def collect(r, enc, info):
            pn = info["pnum"]
            got = [enc.read(pn, OUTPUT, c) for c in range(3)] + [enc.read(pn, QINDEX, 0)]
            mv = enc.read(pn, MV)
            with lock:
                out[(r.name, pn)] = got + ([mv] if mv is not None else [])

        loop = ServingLoop(budget_bytes=int(8e9), max_active=max_active, frame_interval=0.004, collect=collect,
                           batch_me=batch_me)
        return out, loop.run(reqs)

    alone, _ = run(1, False)
    shared, stats = run(4, True)
    assert alone.keys() == shared.keys() and len(alone) == 40
    for k in alone:
        assert len(alone[k]) == len(shared[k]), k
        for a, b in zip(alone[k], shared[k]):
            np.testing.assert_array_equal(a, b, err_msg=str(k))
    est = stats["shared_estimation"]
    assert est["estimates"] > 0 and est["streams_per_round"] > 1.0, est
