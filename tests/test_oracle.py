"""The CPU oracle (oracle/dirac_oracle.c) pinned against the reference codec.

Golden fixtures in tests/golden were produced by running the reference's own C++
(tests/golden/make_golden.py).  Where oracle/_ref is built, the oracle is additionally
checked differentially against the live reference on fresh seeded inputs.
"""
import os

import numpy as np
import pytest

from oracle import Reference


def test_dwt_golden_forward_and_backward(oracle, golden):
    g = golden("dwt.npz")
    metas = [k[:-5] for k in g.files if k.endswith("_meta")]
    assert len(metas) == 21
    for key in metas:
        filt, depth, w, h, cw, ch = (int(v) for v in g[key + "_meta"])
        coeff = oracle.dwt_forward(filt, depth, g[key + "_pic"], cw, ch)
        np.testing.assert_array_equal(coeff, g[key + "_coeff"], err_msg=key)
        back = oracle.dwt_backward(filt, depth, g[key + "_noisy"], w, h)
        np.testing.assert_array_equal(back, g[key + "_back"], err_msg=key)


def test_upconvert_golden(oracle, golden):
    g = golden("convert.npz")
    for k in range(3):
        w, h, bd = (int(v) for v in g[f"up{k}_meta"])
        np.testing.assert_array_equal(oracle.upconvert(g[f"up{k}_pic"], bd), g[f"up{k}_out"])


def test_downconvert_golden(oracle, golden):
    g = golden("convert.npz")
    for k in range(3):
        np.testing.assert_array_equal(oracle.downconvert(g[f"down{k}_pic"]), g[f"down{k}_out"])


def ramp(w, h):
    """The reference unit test's picture: (((i-j) % 13) * 1024) / 13 with C semantics
    (unit_tests/wavelet_utils_test.cpp:50-58)."""
    j, i = np.mgrid[0:h, 0:w]
    d = i - j
    m = np.fmod(d, 13)  # C remainder keeps the dividend's sign
    v = m * 1024
    return (np.sign(v) * (np.abs(v) // 13)).astype(np.int16)  # C division truncates


@pytest.mark.parametrize("filt", range(8))
def test_transform_invertibility_ramp(oracle, filt):
    """Restates unit_tests/wavelet_utils_test.cpp:84-105: 512x512 ramp, depth 1, every
    WltFilter value (FIDELITY and filterNK fall through to DAUB9_7): forward then
    backward returns the input."""
    pic = ramp(512, 512)
    coeff = oracle.dwt_forward(filt, 1, pic)
    np.testing.assert_array_equal(oracle.dwt_backward(filt, 1, coeff, 512, 512), pic)


@pytest.mark.parametrize("filt", range(7))
def test_invertibility_deep(oracle, filt):
    rng = np.random.default_rng(filt)
    pic = rng.integers(-512, 512, size=(77, 131)).astype(np.int16)
    for depth in (2, 4):
        coeff = oracle.dwt_forward(filt, depth, pic)
        np.testing.assert_array_equal(oracle.dwt_backward(filt, depth, coeff, 131, 77), pic)


def test_rejects_undefined_sizes(oracle):
    # a DD filter level side below 6 reads outside the region in the reference
    with pytest.raises(ValueError):
        oracle.dwt_forward(0, 3, np.zeros((16, 16), np.int16))
    with pytest.raises(ValueError):
        oracle.downconvert(np.zeros((22, 40), np.int16))


needs_ref = pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built here")


@needs_ref
@pytest.mark.parametrize("filt", range(7))
def test_dwt_matches_live_reference(oracle, filt):
    ref = Reference()
    rng = np.random.default_rng(100 + filt)
    for (w, h, depth) in [(352, 288, 4), (176, 144, 5), (101, 67, 3), (720, 576, 5)]:
        pic = rng.integers(-128, 128, size=(h, w)).astype(np.int16)
        c_ref = ref.dwt_forward(filt, depth, pic)
        np.testing.assert_array_equal(oracle.dwt_forward(filt, depth, pic), c_ref)
        noisy = (c_ref + rng.integers(-20, 21, size=c_ref.shape)).astype(np.int32)
        np.testing.assert_array_equal(oracle.dwt_backward(filt, depth, noisy, w, h),
                                      ref.dwt_backward(filt, depth, noisy, w, h))


@needs_ref
def test_convert_matches_live_reference(oracle):
    ref = Reference()
    rng = np.random.default_rng(3)
    for (w, h, bd) in [(352, 288, 8), (176, 144, 10), (960, 540, 8)]:
        pic = rng.integers(-(1 << (bd - 1)), 1 << (bd - 1), size=(h, w)).astype(np.int16)
        np.testing.assert_array_equal(oracle.upconvert(pic, bd), ref.upconvert(pic, bd))
        np.testing.assert_array_equal(oracle.downconvert(pic), ref.downconvert(pic))


def mc_case(g, k):
    from oracle import BlockParams

    w, h, cf, prec, xbl, ybl, xbs, ybs, xsb, ysb, nref = (int(v) for v in g[f"mc{k}_meta"])
    bp = BlockParams(prec, xbl, ybl, xbs, ybs, xsb, ysb)
    arrs = {n: g[f"mc{k}_{n}"] for n in ("mv1", "mv2", "mode", "dc", "split")}
    pic = [g[f"mc{k}_pic{c}"] for c in range(3)]
    r1 = [g[f"mc{k}_r1_{c}"] for c in range(3)]
    r2 = [g[f"mc{k}_r2_{c}"] for c in range(3)] if nref == 2 else None
    outs = {aos: [g[f"mc{k}_out{aos}_{c}"] for c in range(3)] for aos in (0, 1)}
    arrs["weights"] = tuple(int(x) for x in g[f"mc{k}_wt"])
    return cf, bp, arrs, pic, r1, r2, outs


MC_GOLDEN_CASES = 8  # 4 with the default reference weights, then 4 with custom ones


def test_motion_compensation_golden(oracle, golden):
    g = golden("mc.npz")
    for k in range(MC_GOLDEN_CASES):
        cf, bp, a, pic, r1, r2, outs = mc_case(g, k)
        bd = 8 if a["weights"] == (1, 1, 1) else 10
        for aos in (0, 1):
            res = oracle.motion_compensate(aos, cf, pic, r1, r2, bp, a["mv1"], a["mv2"], a["mode"], a["dc"],
                                           a["split"], bd, bd, a["weights"])
            for c in range(3):
                np.testing.assert_array_equal(res[c], outs[aos][c], err_msg=f"case {k} aos {aos} comp {c}")


@needs_ref
def test_motion_compensation_matches_live_reference(oracle):
    from oracle import BlockParams, chroma_shift

    ref = Reference()
    rng = np.random.default_rng(77)
    for trial in range(12):
        cf, prec = trial % 3, trial % 4
        w, h = [(352, 288), (176, 144), (120, 72)][trial % 3]
        xbl, ybl, xbs, ybs = [(12, 12, 8, 8), (16, 16, 12, 12), (24, 24, 16, 16), (8, 8, 8, 8)][trial % 4]
        xsb, ysb = (w + 4 * xbs - 1) // (4 * xbs), (h + 4 * ybs - 1) // (4 * ybs)
        bp = BlockParams(prec, xbl, ybl, xbs, ybs, xsb, ysb)
        nb = (4 * ysb, 4 * xsb)
        mv1 = rng.integers(-60 << prec, 60 << prec, size=nb + (2,)).astype(np.int16)
        mv2 = rng.integers(-60 << prec, 60 << prec, size=nb + (2,)).astype(np.int16)
        mode = rng.integers(0, 4, size=nb).astype(np.uint8)
        dc = rng.integers(-128, 128, size=(3,) + nb).astype(np.int16)
        split = rng.integers(0, 3, size=(ysb, xsb)).astype(np.uint8)
        xs, ys = chroma_shift(cf)
        mk = lambda: [rng.integers(-128, 128, size=(h, w)).astype(np.int16)] + [
            rng.integers(-128, 128, size=(h >> ys, w >> xs)).astype(np.int16) for _ in range(2)]
        pic, r1, r2 = mk(), mk(), mk()
        for aos in (0, 1):
            a = oracle.motion_compensate(aos, cf, pic, r1, r2, bp, mv1, mv2, mode, dc, split)
            b = ref.motion_compensate(aos, cf, pic, r1, r2, bp, mv1, mv2, mode, dc, split)
            for c in range(3):
                np.testing.assert_array_equal(a[c], b[c])


# reference picture weights (ref1, ref2, precision bits) of the weighted-compensation checks:
# the precision 0 whose rounding bias the reference leaves at 1, a negative and a zero weight,
# and weights large enough to wrap the reference's int16 block values
MC_WEIGHTS = [(1, 1, 0), (3, 5, 3), (-2, 7, 2), (0, 4, 2), (2, 2, 1), (255, 1, 8), (40, -9, 5)]


@needs_ref
@pytest.mark.parametrize("weights", MC_WEIGHTS, ids=[str(w) for w in MC_WEIGHTS])
def test_weighted_motion_compensation_matches_live_reference(oracle, weights):
    """Custom reference picture weights (AdjustBlockByRefWeights, mot_comp.cpp:620-680): the
    oracle equals the reference's CompensatePicture with the weights set in its
    PicturePredParams, on every prediction mode, both directions and all chroma formats."""
    from oracle import BlockParams, chroma_shift

    ref = Reference()
    rng = np.random.default_rng(78 + sum(abs(x) for x in weights))
    for trial in range(3):
        cf, prec = trial, (trial + 1) % 4
        w, h = [(176, 144), (120, 72), (96, 64)][trial]
        xbl, ybl, xbs, ybs = [(12, 12, 8, 8), (16, 16, 12, 12), (8, 8, 8, 8)][trial]
        xsb, ysb = (w + 4 * xbs - 1) // (4 * xbs), (h + 4 * ybs - 1) // (4 * ybs)
        bp = BlockParams(prec, xbl, ybl, xbs, ybs, xsb, ysb)
        nb = (4 * ysb, 4 * xsb)
        mv1 = rng.integers(-40 << prec, 40 << prec, size=nb + (2,)).astype(np.int16)
        mv2 = rng.integers(-40 << prec, 40 << prec, size=nb + (2,)).astype(np.int16)
        mode = rng.integers(0, 4, size=nb).astype(np.uint8)
        dc = rng.integers(-512, 512, size=(3,) + nb).astype(np.int16)
        split = rng.integers(0, 3, size=(ysb, xsb)).astype(np.uint8)
        xs, ys = chroma_shift(cf)
        mk = lambda: [rng.integers(-512, 512, size=(h, w)).astype(np.int16)] + [
            rng.integers(-512, 512, size=(h >> ys, w >> xs)).astype(np.int16) for _ in range(2)]
        pic, r1, r2 = mk(), mk(), mk()
        for aos in (0, 1):
            a = oracle.motion_compensate(aos, cf, pic, r1, r2, bp, mv1, mv2, mode, dc, split, 10, 10, weights)
            b = ref.motion_compensate(aos, cf, pic, r1, r2, bp, mv1, mv2, mode, dc, split, 10, 10, weights)
            for c in range(3):
                np.testing.assert_array_equal(a[c], b[c], err_msg=f"trial {trial} aos {aos} comp {c}")
            if weights != (1, 1, 1):
                d = oracle.motion_compensate(aos, cf, pic, r1, r2, bp, mv1, mv2, mode, dc, split, 10, 10)
                assert any(not np.array_equal(a[c], d[c]) for c in range(3))


def me_case(g, k):
    from oracle import BlockParams

    w, h, cf, prec, xbl, ybl, xbs, ybs, xsb, ysb, nref = (int(v) for v in g[f"me{k}_meta"])
    bp = BlockParams(prec, xbl, ybl, xbs, ybs, xsb, ysb)
    pic = [g[f"me{k}_pic{c}"] for c in range(3)]
    r1 = [g[f"me{k}_r1_{c}"] for c in range(3)]
    r2 = [g[f"me{k}_r2_{c}"] for c in range(3)] if nref == 2 else None
    want = {n: g[f"me{k}_{n}"] for n in ("mv", "cost", "mode", "dc", "split", "sbcost")}
    return cf, bp, pic, r1, r2, float(g[f"me{k}_lambda"][0]), want


def test_motion_estimation_golden(oracle, golden):
    g = golden("me.npz")
    for k in range(3):
        cf, bp, pic, r1, r2, lam, want = me_case(g, k)
        got = oracle.motion_estimate(cf, pic, r1, r2, bp, lam, 3)
        for n, a in want.items():
            np.testing.assert_array_equal(got[n], a, err_msg=f"case {k} {n}")


def test_me_depth_formula(oracle):
    # (int)min(log2(W/12), log2(H/12)) (libdirac_motionest/pixel_match.cpp:94-95)
    assert oracle.me_depth(352, 288) == 4
    assert oracle.me_depth(1920, 1080) == 6
    assert oracle.me_depth(3840, 2160) == 7


@needs_ref
@pytest.mark.parametrize("case", range(6))
def test_motion_estimation_matches_live_reference(oracle, case):
    import sys

    from oracle import BlockParams

    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "dirac-research_b200"))
    from dirac_b200 import synth

    w, h, olb, prec, nref, chroma, vmax = [
        (352, 288, (12, 12, 8, 8), 2, 2, "420", 8), (352, 288, (12, 12, 8, 8), 2, 1, "420", 8),
        (720, 576, (12, 12, 8, 8), 3, 2, "422", 16), (480, 272, (16, 16, 12, 12), 1, 2, "444", 12),
        (960, 540, (16, 16, 12, 12), 2, 2, "420", 24), (640, 360, (24, 24, 16, 16), 2, 2, "420", 24)][case]
    seq = synth.make_sequence(w, h, 3, n_rects=12, vmax=vmax, seed=900 + case, chroma=chroma)
    f = [[synth.to_signed(p) for p in fr] for fr in seq]
    xbl, ybl, xbs, ybs = olb
    bp = BlockParams(prec, xbl, ybl, xbs, ybs, (w + 4 * xbs - 1) // (4 * xbs), (h + 4 * ybs - 1) // (4 * ybs))
    cf = {"444": 0, "422": 1, "420": 2}[chroma]
    lam = float(2 * np.sqrt(4 * 10 ** ((12 - 7) / 2.5) / 16))
    a = oracle.motion_estimate(cf, f[1], f[0], f[2] if nref == 2 else None, bp, lam, 3)
    b = Reference().motion_estimate(cf, f[1], f[0], f[2] if nref == 2 else None, bp, lam, 3)
    for n in a:
        np.testing.assert_array_equal(a[n], b[n], err_msg=n)


def quant_case(g, k):
    w, h, depth, filt, intra, comp = (int(v) for v in g[f"q{k}_meta"])
    names = ("recon", "qidx", "skip", "wt", "ecf", "bits", "ncb", "cb_skip")
    return (w, h, depth, filt, intra, comp, float(g[f"q{k}_lambda"][0]), g[f"q{k}_coeff"],
            {n: g[f"q{k}_{n}"] for n in names})


def test_code_residue_golden(oracle, golden):
    g = golden("quant.npz")
    for k in range(4):
        w, h, depth, filt, intra, comp, lam, coeff, want = quant_case(g, k)
        recon, q, sk, bits, cbs, _ = oracle.code_residue(intra, depth, coeff, lam, want["wt"].astype(np.float32),
                                                         want["ecf"], want["ncb"])
        np.testing.assert_array_equal(recon, want["recon"], err_msg=f"case {k}")
        np.testing.assert_array_equal(sk, want["skip"])
        np.testing.assert_array_equal(q[sk == 0], want["qidx"][sk == 0])
        np.testing.assert_array_equal(bits, want["bits"])
        np.testing.assert_array_equal(cbs, want["cb_skip"])


def test_quantiser_factor_table(oracle):
    from dirac_b200 import _lib

    lib = _lib.load()
    # QuantiserLists: qf4[0]=4, qf4[1]=5, then 4 * 2^(q/4) with fixed rational steps
    assert [lib.dgpu_quant_factor4(q) for q in range(8)] == [4, 5, 6, 7, 8, 10, 11, 13]
    assert lib.dgpu_quant_factor4(40) == 4096
    assert [lib.dgpu_quant_factor4(q) for q in range(120)] == [oracle.lib.orc_qf4(q) for q in range(120)]


def test_band_weights_and_code_blocks_match_reference_fixtures(golden):
    """Host helpers dgpu_band_weights / dgpu_code_blocks reproduce the reference's
    SetBandWeights and code-block grid (the fixtures hold the reference's values; CPD 20, the
    default video format's)."""
    from dirac_b200 import quant

    g = golden("quant.npz")
    for k in range(4):
        w, h, depth, filt, intra, comp, lam, coeff, want = quant_case(g, k)
        ch, cw = coeff.shape
        wt = quant.band_weights(filt, depth, cw, ch, comp, 2, 20.0, 1.0)
        np.testing.assert_array_equal(wt, want["wt"], err_msg=f"case {k}")
        np.testing.assert_array_equal(quant.code_blocks(depth, w, h), want["ncb"])


@needs_ref
@pytest.mark.parametrize("case", range(6))
def test_code_residue_matches_live_reference(oracle, case):
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "dirac-research_b200"))
    from dirac_b200 import quant, synth

    w, h, depth, filt, intra, comp, qf, cf = [(352, 288, 4, 6, 1, 0, 7, 2), (352, 288, 4, 0, 0, 1, 7, 2),
                                              (720, 576, 5, 2, 1, 0, 5, 1), (720, 576, 4, 1, 0, 2, 9, 2),
                                              (1920, 1080, 4, 6, 1, 0, 7, 2), (1280, 720, 3, 3, 0, 0, 6, 2)][case]
    seq = synth.make_sequence(w, h, 2, n_rects=12, vmax=12, seed=300 + case,
                              chroma={2: "420", 1: "422", 0: "444"}[cf])
    f = [synth.to_signed(p) for p in seq[0]]
    g = [synth.to_signed(p) for p in seq[1]]
    pic = f[comp] if intra else np.clip(f[comp].astype(np.int32) - g[comp], -128, 127).astype(np.int16)
    coeff = oracle.dwt_forward(filt, depth, pic)
    lam = 10 ** ((12 - qf) / 2.5) / 16 * (1 if intra else 4)
    r = Reference().code_residue(cf, w, h, comp, intra, filt, depth, coeff, lam)
    ch, cw = coeff.shape
    np.testing.assert_array_equal(quant.band_weights(filt, depth, cw, ch, comp, cf, 20.0, 1.0), r["wt"])
    np.testing.assert_array_equal(quant.code_blocks(depth, w, h), r["ncb"])
    recon, q, sk, bits, cbs, _ = oracle.code_residue(intra, depth, coeff, lam, r["wt"].astype(np.float32), r["ecf"],
                                                     r["ncb"])
    np.testing.assert_array_equal(recon, r["recon"])
    np.testing.assert_array_equal(sk, r["skip"])
    np.testing.assert_array_equal(q[sk == 0], r["qidx"][sk == 0])
    np.testing.assert_array_equal(bits, r["bits"])
    np.testing.assert_array_equal(cbs, r["cb_skip"])
