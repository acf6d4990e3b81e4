"""The host arithmetic coder of quantised subbands (dgpu_code_bands_host) and the
entropy-correction factors (dgpu_entropy_*) against the reference, without a GPU.

Band data: for seeded components (intra and inter, several filters, depths and sizes) the
coder, given the oracle's quantised indices for the reference's quantiser choices, writes the
bytes the reference's band coders write, arithmetic and variable-length (tests/golden/bands.npz: CRC-32 and length of every
band's data, made through the reference's own BandCodec / IntraDCBandCodec; live comparison
where oracle/_ref exists).  Whole loop: the oracle's restated coding loop, with the
entropy-correction factors adapted from this coder's byte counts, reproduces the stock
reference encoder (adaptive factors, as it ships), with arithmetic and with variable-length
coefficient coding, picture for picture (tests/golden/adaptive.npz)."""
import os
import sys
import zlib

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import BAND_CASES, ENCODE_CASES, encode_inputs  # noqa: E402


def band_inputs(oracle, golden, k):
    intra, filt, depth, w, h, lam = BAND_CASES[k]
    g = golden("bands.npz")
    rng = np.random.default_rng(900 + k)
    pic = rng.integers(-60, 60, size=(h, w)).astype(np.int16)
    co = oracle.dwt_forward(filt, depth, pic)
    _, q, sk, bits, cbs, qo = oracle.code_residue(intra, depth, co, lam, g[f"c{k}_wt"].astype(np.float32),
                                                  g[f"c{k}_ecf"], g[f"c{k}_ncb"])
    return intra, depth, q, sk, cbs, qo, g


def _adversarial_indices(kind, rng, cw=128, ch=96):
    """Index arrays that stress the range coder: no symbols, long follow-bit codes, symbols near
    even odds (long runs of deferred bits), isolated large values, whole zero code blocks."""
    if kind == "zero":
        return np.zeros((ch, cw), np.int32)
    if kind == "huge":
        return rng.integers(-(1 << 20), 1 << 20, size=(ch, cw)).astype(np.int32)
    if kind == "signs":
        return rng.choice(np.array([-1, 1], np.int32), size=(ch, cw))
    if kind == "even":
        return rng.integers(-2, 3, size=(ch, cw)).astype(np.int32)
    if kind == "sparse":
        q = np.zeros((ch, cw), np.int32)
        m = rng.random((ch, cw)) < 0.02
        q[m] = (rng.geometric(0.05, size=int(m.sum())) * rng.choice([-1, 1], size=int(m.sum()))).astype(np.int32)
        return q
    if kind == "blocks":
        q = rng.integers(-40, 41, size=(ch, cw)).astype(np.int32)
        q[(np.arange(ch)[:, None] // 8 + np.arange(cw)[None, :] // 8) % 3 == 0] = 0
        return q
    if kind == "stripes":
        q = np.zeros((ch, cw), np.int32)
        q[::2, :] = np.where(np.arange(cw) % 2 == 0, 5, -5)
        q[:, ::3] = -np.arange(ch)[:, None] % 7
        return q
    raise ValueError(kind)


@pytest.mark.parametrize("kind", ["zero", "huge", "signs", "even", "sparse", "blocks", "stripes"])
def test_band_coder_matches_reference_on_adversarial_indices(kind):
    """The range coder's bytes equal the reference band coders' own on index arrays chosen to
    stress it (the reference coding given indices at quantiser index 0, inter bands), with one
    code block per band and with several, some skipped."""
    from oracle import Reference

    from dirac_b200.entropy import code_bands

    if not Reference.available():
        pytest.skip("reference library not built here")
    ref = Reference()
    depth = 4
    rng = np.random.default_rng(sum(map(ord, kind)))
    q = _adversarial_indices(kind, rng)
    for ncb in (np.ones((3 * depth + 1, 2), np.int32),
                np.array([[1, 1]] * 4 + [[2, 2]] * 3 + [[4, 3]] * 3 + [[3, 4]] * 3, np.int32)[::-1].copy()):
        want, want_bytes, cbs = ref.code_inter_indices_bytes(depth, q, ncb)
        bands = np.zeros((3 * depth + 1, 3), np.int32)
        data, per = code_bands(0, depth, [q], [bands], [ncb], [cbs])
        np.testing.assert_array_equal(per[0], want_bytes, err_msg=kind)
        assert data.tobytes() == want.tobytes(), kind


_POOL_SNIPPET = """
import sys, zlib
import numpy as np
sys.path.insert(0, sys.argv[1])
from dirac_b200 import quant
from dirac_b200.entropy import code_bands
rng = np.random.default_rng(77)
depth, cw, ch = 3, 128, 96
q = rng.integers(-40, 41, size=(ch, cw)).astype(np.int32)
q[rng.random((ch, cw)) < 0.7] = 0
ncb = np.asarray(quant.code_blocks(depth, cw, ch), np.int32).reshape(-1, 2)
bands = np.zeros((3 * depth + 1, 2), np.int32)
cbs = np.zeros(int((ncb[:, 0] * ncb[:, 1]).sum()), np.uint8)
data, per = code_bands(0, depth, [q, q[::-1].copy(), -q], [bands] * 3, [ncb] * 3, [cbs] * 3)
print(zlib.crc32(data.tobytes()), [int(x) for p in per for x in p])
"""


@pytest.mark.parametrize("threads", ["1", "3"])
def test_host_pool_size_variable(threads):
    """DGPU_HOST_THREADS sizes the library's host pool when it is first used: the coded bands do
    not depend on it (a fresh process per setting, against the default pool)."""
    import subprocess

    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "dirac-research_b200")
    run = lambda env: subprocess.run([sys.executable, "-c", _POOL_SNIPPET, pkg], env=env, capture_output=True,  # noqa: E731
                                     text=True, timeout=120, check=True).stdout
    base = {k: v for k, v in os.environ.items() if k != "DGPU_HOST_THREADS"}
    assert run(dict(base, DGPU_HOST_THREADS=threads)) == run(base)


@pytest.mark.parametrize("k", range(len(BAND_CASES)))
def test_band_data_matches_reference_fixture(oracle, golden, k):
    from dirac_b200.entropy import code_bands

    intra, depth, q, sk, cbs, qo, g = band_inputs(oracle, golden, k)
    np.testing.assert_array_equal(sk, g[f"c{k}_skip"])
    np.testing.assert_array_equal(q[sk == 0], g[f"c{k}_qidx"][sk == 0])
    np.testing.assert_array_equal(cbs, g[f"c{k}_cb_skip"])
    data, per = code_bands(intra, depth, [qo], [np.stack([q, sk], 1)], [g[f"c{k}_ncb"]], [cbs])
    np.testing.assert_array_equal(per[0], g[f"c{k}_band_bytes"])
    crc, start = [], 0
    for b in range(3 * depth + 1, 0, -1):
        n = int(per[0][b - 1])
        crc.append(zlib.crc32(data[start:start + n].tobytes()))
        start += n
    np.testing.assert_array_equal(np.array(crc[::-1], np.uint32), g[f"c{k}_band_crc"])
    # the same indices as int16 (dgpu_code_bands_host16): the same bytes
    assert np.abs(qo).max() <= 32767
    data16, per16 = code_bands(intra, depth, [qo.astype(np.int16)], [np.stack([q, sk], 1)], [g[f"c{k}_ncb"]],
                               [cbs])
    np.testing.assert_array_equal(per16[0], per[0])
    np.testing.assert_array_equal(data16, data)


@pytest.mark.parametrize("k", range(len(BAND_CASES)))
def test_vlc_band_data_matches_reference_fixture(oracle, golden, k):
    """The variable-length form (dgpu_code_bands_vlc_host) against the reference's BandVLC /
    IntraDCBandVLC: bytes, lengths, and the whole-byte counts its Compress returns."""
    from dirac_b200.entropy import code_bands

    intra, depth, q, sk, cbs, qo, g = band_inputs(oracle, golden, k)
    data, per, bits = code_bands(intra, depth, [qo], [np.stack([q, sk], 1)], [g[f"c{k}_ncb"]], [cbs], vlc=True)
    np.testing.assert_array_equal(per[0], g[f"c{k}_vlc_band_bytes"])
    np.testing.assert_array_equal(bits[0] // 8, g[f"c{k}_vlc_compress_bytes"])
    crc, start = [], 0
    for b in range(3 * depth + 1, 0, -1):
        n = int(per[0][b - 1])
        crc.append(zlib.crc32(data[start:start + n].tobytes()))
        start += n
    np.testing.assert_array_equal(np.array(crc[::-1], np.uint32), g[f"c{k}_vlc_band_crc"])


def test_band_data_matches_live_reference(oracle):
    from dirac_b200.entropy import code_bands
    from oracle import Reference

    if not Reference.available():
        pytest.skip("reference library not built here")
    ref = Reference()
    rng = np.random.default_rng(77)
    for intra, filt, depth, w, h, lam, comp in [(1, 0, 4, 160, 96, 2.0, 1), (0, 6, 3, 120, 72, 12.0, 2)]:
        pic = rng.integers(-90, 90, size=(h, w)).astype(np.int16)
        co = oracle.dwt_forward(filt, depth, pic)
        r = ref.code_residue_bytes(2, 2 * w if comp else w, 2 * h if comp else h, comp, intra, filt, depth, co, lam)
        _, q, sk, _, cbs, qo = oracle.code_residue(intra, depth, co, lam, r["wt"].astype(np.float32), r["ecf"],
                                                   r["ncb"])
        data, per = code_bands(intra, depth, [qo], [np.stack([q, sk], 1)], [r["ncb"]], [cbs])
        np.testing.assert_array_equal(per[0], r["band_bytes"])
        np.testing.assert_array_equal(data, r["data"])
        v = ref.code_residue_vlc_bytes(2, 2 * w if comp else w, 2 * h if comp else h, comp, intra, filt, depth, co,
                                       lam)
        vdata, vper, _ = code_bands(intra, depth, [qo], [np.stack([q, sk], 1)], [r["ncb"]], [cbs], vlc=True)
        np.testing.assert_array_equal(vper[0], v["band_bytes"])
        np.testing.assert_array_equal(vdata, v["data"])


def adaptive_encode(case, vlc=False):
    """The oracle's coding loop with factors adapted from the host coder's byte counts
    (dgpu_code_bands_host; with vlc, dgpu_code_bands_vlc_host and the whole bytes the
    reference's VLC coders report)."""
    from dirac_b200 import quant, synth
    from dirac_b200.entropy import EntropyCorrector, code_bands
    from oracle_encoder import OracleEncoder

    seq, rcfg = encode_inputs(case)
    cfg = {k: v for k, v in rcfg.items() if k != "video_format"}
    cfg.update(luma_depth=8, chroma_depth=8)
    depth = cfg["wlt_depth"]
    ec = EntropyCorrector(depth)
    enc = OracleEncoder(cfg, quant.band_weights, quant.code_blocks, ecf_fn=lambda p: ec.factors(p.intra, p.is_b()))
    for f in seq:
        enc.load([synth.to_signed(x) for x in f])
    enc.end_sequence()
    ncb = quant.code_blocks(depth, cfg["width"], cfg["height"])
    while True:
        p = enc.code_next()
        if p is None:
            break
        r = p.result
        for c in range(3):
            coded = code_bands(p.intra, depth, [r["qindex"][c]], [np.stack([r["qidx"][c], r["skip"][c]], 1)], [ncb],
                               [r["cb_skip"][c]], vlc=vlc)
            counts = coded[2][0] // 8 if vlc else coded[1][0]
            ec.update(p.intra, p.is_b(), c, r["skip"][c], r["bits"][c], counts)
    return enc


@pytest.mark.parametrize("case", ENCODE_CASES, ids=[c[0] for c in ENCODE_CASES])
def test_adaptive_loop_matches_stock_reference_encoder(golden, case):
    enc = adaptive_encode(case)
    g = golden("adaptive.npz")
    crc = np.array([[zlib.crc32(np.ascontiguousarray((p.astype(np.int32) + 128).astype(np.uint8)).tobytes())
                     for p in enc.pics[i].data] for i in range(len(enc.pics))], np.uint32)
    np.testing.assert_array_equal(crc, g[case[0] + "_crc"])
    np.testing.assert_array_equal([int(enc.pics[i].intra) for i in range(len(enc.pics))], g[case[0] + "_ptype"])
    # the adapted factors matter: the stock encoder's pictures differ from the frozen-factor ones
    assert not np.array_equal(g[case[0] + "_crc"], golden("encode.npz")[case[0] + "_crc"])


@pytest.mark.parametrize("case", ENCODE_CASES, ids=[c[0] for c in ENCODE_CASES])
def test_adaptive_vlc_loop_matches_stock_reference_encoder(golden, case):
    """The same with variable-length coefficient coding (-use_vlc): the stock reference
    encoder's pictures."""
    enc = adaptive_encode(case, vlc=True)
    g = golden("adaptive.npz")
    crc = np.array([[zlib.crc32(np.ascontiguousarray((p.astype(np.int32) + 128).astype(np.uint8)).tobytes())
                     for p in enc.pics[i].data] for i in range(len(enc.pics))], np.uint32)
    np.testing.assert_array_equal(crc, g[case[0] + "_vlc_crc"])
    np.testing.assert_array_equal([int(enc.pics[i].intra) for i in range(len(enc.pics))], g[case[0] + "_vlc_ptype"])


@pytest.mark.parametrize("depth", [1, 3, 4, 6])
def test_entropy_corrector_initial_factors(depth):
    from dirac_b200.entropy import EntropyCorrector
    from oracle_encoder import initial_ecf

    ec = EntropyCorrector(depth)
    for intra, is_b in [(1, 0), (0, 1), (0, 0)]:
        f = ec.factors(intra, is_b)
        for c in range(3):
            np.testing.assert_array_equal(f[c], initial_ecf(depth, bool(intra)))


def test_entropy_corrector_update_rule():
    """EntropyCorrector::Update: factor *= float(actual bits) / float(estimated bits), for the
    picture kind (intra, B, other inter) and component given; skipped bands unchanged; a zero
    count leaves the factor alone."""
    from dirac_b200.entropy import EntropyCorrector

    ec = EntropyCorrector(1)
    before = ec.factors(0, 1).copy()
    ec.update(0, 1, 2, [0, 1, 0, 0], [100, 100, 0, 80], [25, 25, 25, 0])
    after = ec.factors(0, 1)
    np.testing.assert_array_equal(after[:2], before[:2])
    assert after[2, 0] == np.float32(before[2, 0] * np.float32(np.float32(200) / np.float32(100)))
    assert after[2, 1] == before[2, 1] and after[2, 2] == before[2, 2] and after[2, 3] == before[2, 3]
    np.testing.assert_array_equal(ec.factors(0, 0), EntropyCorrector(1).factors(0, 0))


def test_code_bands_reports_size():
    """A too-small output buffer returns DGPU_ERR_SIZE with every band's length filled."""
    import ctypes

    from dirac_b200 import _lib

    q = np.zeros((8, 8), np.int32)
    q[0, 0] = 3
    n = np.zeros(4, np.int32)
    out = np.zeros(1, np.uint8)
    rc = _lib.load().dgpu_code_bands_host(
        1, _lib.int_array([1]), _lib.int_array([1]), _lib.ptr_array([q.ctypes.data]), _lib.int_array([8]),
        _lib.int_array([8]), _lib.int_array([1, 1] * 4), _lib.int_array([0] * 4), _lib.int_array([0] * 4),
        np.zeros(4, np.uint8).ctypes.data, out.ctypes.data, ctypes.c_size_t(0), n.ctypes.data_as(_lib.P_int))
    assert rc == -2 and (n > 0).all()


@pytest.mark.parametrize("vlc", [False, True], ids=["ac", "vlc"])
def test_decode_bands_round_trip(oracle, golden, vlc):
    """dgpu_decode_bands_host inverts the coder (whose bytes are the reference's, above)."""
    from dirac_b200.entropy import code_bands, decode_bands

    for k in range(len(BAND_CASES)):
        intra, depth, q, sk, cbs, qo, g = band_inputs(oracle, golden, k)
        coded = code_bands(intra, depth, [qo], [np.stack([q, sk], 1)], [g[f"c{k}_ncb"]], [cbs], vlc=vlc)
        got, flags = decode_bands(depth, [qo.shape], [sk], [g[f"c{k}_ncb"]], coded[0], [coded[1][0]], vlc=vlc)
        np.testing.assert_array_equal(got[0], qo, err_msg=f"case {k}")
        np.testing.assert_array_equal(flags[0], cbs, err_msg=f"case {k}")


def test_decode_bands_of_live_reference_bytes(oracle):
    """The reference band coders' own bytes decode to the indices the oracle quantises to."""
    from dirac_b200.entropy import decode_bands
    from oracle import Reference

    if not Reference.available():
        pytest.skip("reference library not built here")
    ref = Reference()
    rng = np.random.default_rng(31)
    for intra, filt, depth, w, h, lam in [(1, 6, 4, 176, 144, 4.0), (0, 0, 3, 120, 72, 25.0)]:
        pic = rng.integers(-70, 70, size=(h, w)).astype(np.int16)
        co = oracle.dwt_forward(filt, depth, pic)
        for vlc in (False, True):
            r = (ref.code_residue_vlc_bytes if vlc else ref.code_residue_bytes)(2, w, h, 0, intra, filt, depth, co,
                                                                                 lam)
            _, q, sk, _, cbs, qo = oracle.code_residue(intra, depth, co, lam, r["wt"].astype(np.float32), r["ecf"],
                                                       r["ncb"])
            got, flags = decode_bands(depth, [qo.shape], [r["skip"]], [r["ncb"]], r["data"], [r["band_bytes"]],
                                      vlc=vlc)
            np.testing.assert_array_equal(got[0], qo)
            np.testing.assert_array_equal(flags[0], cbs)


def test_coded_bytes_decode_to_the_reference_decoders_pictures(oracle, golden):
    """From coded band bytes to pictures: a sequence's bands coded, decoded back to indices and
    flags, and decoded by the oracle's restatement of the decoder, give the reference decoder's
    pictures (decode.npz)."""
    from dirac_b200 import quant, synth
    from dirac_b200.entropy import code_bands, decode_bands
    from oracle_decoder import decode_picture, output_samples
    from oracle_encoder import encode_sequence

    seq, rcfg = encode_inputs(ENCODE_CASES[1])
    cfg = {k: v for k, v in rcfg.items() if k != "video_format"}
    cfg.update(luma_depth=8, chroma_depth=8)
    enc = encode_sequence(cfg, [[synth.to_signed(x) for x in f] for f in seq], quant.band_weights, quant.code_blocks,
                          oracle)
    depth = cfg["wlt_depth"]
    ncb = quant.code_blocks(depth, cfg["width"], cfg["height"])
    out = {}
    for pn in enc.order:
        p = enc.pics[pn]
        r = p.result
        shapes = [x.shape for x in r["qindex"]]
        bands = [np.stack([r["qidx"][c], r["skip"][c]], 1) for c in range(3)]
        data, per = code_bands(p.intra, depth, r["qindex"], bands, [ncb] * 3, r["cb_skip"])
        q, flags = decode_bands(depth, shapes, r["skip"], [ncb] * 3, data, per)
        pic = {"intra": p.intra, "filter": r["filter"], "qindex": q, "qidx": r["qidx"], "skip": r["skip"],
               "cb_skip": flags, "me": p.me}
        out[pn] = decode_picture(cfg, pic, [out[x] for x in p.refs] if not p.intra else None, ncb, oracle)
    crc = np.array([[zlib.crc32(np.ascontiguousarray(x).tobytes()) for x in output_samples(out[i], 8, 8)]
                    for i in range(len(seq))], np.uint32)
    np.testing.assert_array_equal(crc, golden("decode.npz")[ENCODE_CASES[1][0] + "_crc"])


@pytest.mark.parametrize("vlc", [False, True], ids=["ac", "vlc"])
def test_round_trip_extreme_indices(vlc):
    """Magnitudes up to 2^30, all-zero bands, empty code blocks (more blocks than samples) and
    a single-block band survive coding and decoding."""
    from dirac_b200.entropy import code_bands, decode_bands

    rng = np.random.default_rng(41)
    depth, cw, ch = 3, 40, 24
    nb = 3 * depth + 1
    q = np.zeros((ch, cw), np.int32)
    mask = rng.random((ch, cw)) < 0.3
    q[mask] = rng.integers(-(1 << 30), 1 << 30, size=int(mask.sum()))
    q[:ch // 8, :cw // 8] = 0  # an all-zero DC band
    ncb = np.array([[7, 5]] * (nb - 1) + [[1, 1]], np.int32)  # band 1 is 20 x 12: fine; DC band 5 x 3: one block
    ncb[nb - 4] = [9, 4]  # a coarse band (5 x 3) with more code blocks than columns: some are empty
    cbs = (rng.random(int((ncb[:, 0] * ncb[:, 1]).sum())) < 0.2).astype(np.uint8)
    # skipped code blocks hold zero indices, as the quantiser writes them
    start = 0
    for b in range(1, nb + 1):
        xn, yn = ncb[b - 1]
        level = (b - 1) // 3 + 1
        if b == nb:
            xp = yp = 0
            xl, yl = cw >> depth, ch >> depth
        else:
            xl, yl = cw >> level, ch >> level
            kind = (b - 1) % 3
            xp = xl if kind in (0, 2) else 0
            yp = yl if kind in (0, 1) else 0
        for by in range(yn):
            for bx in range(xn):
                if cbs[start + by * xn + bx]:
                    q[yp + by * yl // yn:yp + (by + 1) * yl // yn, xp + bx * xl // xn:xp + (bx + 1) * xl // xn] = 0
        if xn * yn == 1:
            cbs[start] = 0
        start += xn * yn
    skip = np.zeros(nb, np.int32)
    skip[2] = 1  # a skipped band: its indices are zero
    xl, yl = cw >> 1, ch >> 1
    q[0:yl, xl:2 * xl] = 0  # band 3 (level 1, kind 2) sits at (xl, 0)
    s0 = sum(int(ncb[b, 0] * ncb[b, 1]) for b in range(2))
    cbs[s0:s0 + int(ncb[2, 0] * ncb[2, 1])] = 0
    coded = code_bands(1, depth, [q], [np.stack([np.zeros(nb, np.int32), skip], 1)], [ncb], [cbs], vlc=vlc)
    assert coded[1][0][2] == 0
    got, flags = decode_bands(depth, [q.shape], [skip], [ncb], coded[0], [coded[1][0]], vlc=vlc)
    np.testing.assert_array_equal(got[0], q)
    np.testing.assert_array_equal(flags[0], cbs)


@pytest.mark.parametrize("vlc", [False, True])
def test_decoder_rejects_band_lengths_past_the_data(vlc):
    """Band lengths come from the stream's subband headers: when they add up to more than the
    data the caller holds (a truncated or corrupt stream), the decoder refuses before reading."""
    from dirac_b200._lib import DgpuError
    from dirac_b200.entropy import code_bands, decode_bands

    rng = np.random.default_rng(11)
    depth, cw, ch = 2, 32, 32
    q = rng.integers(-20, 21, size=(ch, cw)).astype(np.int32)
    nb = 3 * depth + 1
    ncb = np.ones((nb, 2), np.int32)
    skip = np.zeros(nb, np.int32)
    cbs = np.zeros(nb, np.uint8)
    coded = code_bands(1, depth, [q], [np.stack([np.zeros(nb, np.int32), skip], 1)], [ncb], [cbs], vlc=vlc)
    got, _ = decode_bands(depth, [q.shape], [skip], [ncb], coded[0], [coded[1][0]], vlc=vlc)
    np.testing.assert_array_equal(got[0], q)
    with pytest.raises(DgpuError):
        decode_bands(depth, [q.shape], [skip], [ncb], coded[0][:-1], [coded[1][0]], vlc=vlc)
