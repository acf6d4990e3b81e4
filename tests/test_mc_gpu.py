"""GPU parity of upconversion, decimation and OBMC motion compensation (bit-exact)."""
import numpy as np
import pytest
import torch

from test_oracle import mc_case

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_upconvert_golden_and_oracle(gpu, oracle, golden):
    g = golden("convert.npz")
    for k in range(3):
        w, h, bd = (int(v) for v in g[f"up{k}_meta"])
        np.testing.assert_array_equal(gpu.upconvert(dev(g[f"up{k}_pic"]), bd).cpu().numpy(), g[f"up{k}_out"])
    rng = np.random.default_rng(1)
    for (w, h, bd) in [(1920, 1080, 8), (960, 540, 8), (1280, 720, 10), (352, 288, 8), (33, 17, 10), (8, 8, 8),
                       (721, 9, 8)]:
        pic = rng.integers(-(1 << (bd - 1)), 1 << (bd - 1), size=(h, w)).astype(np.int16)
        np.testing.assert_array_equal(gpu.upconvert(dev(pic), bd).cpu().numpy(), oracle.upconvert(pic, bd),
                                      err_msg=f"{w}x{h}")


def test_downconvert_golden_and_oracle(gpu, oracle, golden):
    g = golden("convert.npz")
    for k in range(3):
        np.testing.assert_array_equal(gpu.downconvert(dev(g[f"down{k}_pic"])).cpu().numpy(), g[f"down{k}_out"])
    rng = np.random.default_rng(2)
    for (w, h) in [(1920, 1080), (960, 540), (480, 270), (60, 33), (24, 24), (25, 31)]:
        pic = rng.integers(-128, 128, size=(h, w)).astype(np.int16)
        np.testing.assert_array_equal(gpu.downconvert(dev(pic)).cpu().numpy(), oracle.downconvert(pic),
                                      err_msg=f"{w}x{h}")


def test_pyramid_1080p_depth6(gpu, oracle):
    """The ME pyramid of a 1080p picture: depth (int)min(log2(W/12), log2(H/12)) = 6
    (libdirac_motionest/pixel_match.cpp:94-95), sizes W/2^l x H/2^l."""
    rng = np.random.default_rng(3)
    pic = rng.integers(-128, 128, size=(1080, 1920)).astype(np.int16)
    cur, t = pic, dev(pic)
    for lev in range(1, 7):
        cur = oracle.downconvert(cur)
        t = gpu.downconvert(t)
        np.testing.assert_array_equal(t.cpu().numpy(), cur, err_msg=f"level {lev}")
        assert cur.shape == (1080 >> lev, 1920 >> lev)


def gpu_mc(gpu, aos, cf, bp, a, pic, r1, r2, clip=(0, 0), lbd=8):
    ups1 = [gpu.upconvert(dev(r), lbd) for r in r1]
    ups2 = [gpu.upconvert(dev(r), lbd) for r in r2] if r2 is not None else None
    p = [dev(x) for x in pic]
    bpg = gpu.BlockParams(bp.precision, bp.xblen, bp.yblen, bp.xbsep, bp.ybsep, bp.xnum_sb, bp.ynum_sb)
    mc = gpu.MotionCompensator(bpg, cf)
    mc.CompensatePicture(aos, dev(a["mv1"]), dev(a["mv2"]), dev(a["mode"]), dev(a["dc"]), dev(a["split"]), p,
                         ups1, ups2, clip_depths=clip, weights=a.get("weights", (1, 1, 1)))
    return [x.cpu().numpy() for x in p]


def test_mc_golden(gpu, golden):
    """The reference's CompensatePicture outputs (mc.npz), with default and custom reference
    picture weights."""
    from test_oracle import MC_GOLDEN_CASES

    g = golden("mc.npz")
    for k in range(MC_GOLDEN_CASES):
        cf, bp, a, pic, r1, r2, outs = mc_case(g, k)
        bd = 8 if a["weights"] == (1, 1, 1) else 10
        for aos in (0, 1):
            res = gpu_mc(gpu, aos, cf, bp, a, pic, r1, r2, lbd=bd)
            for c in range(3):
                np.testing.assert_array_equal(res[c], outs[aos][c], err_msg=f"case {k} aos {aos} comp {c}")


@pytest.mark.parametrize("trial", range(16))
def test_mc_vs_oracle(gpu, oracle, trial):
    from oracle import BlockParams, chroma_shift

    rng = np.random.default_rng(500 + trial)
    cf, prec = trial % 3, trial % 4
    w, h = [(352, 288), (1920, 1080), (176, 144), (130, 98)][trial % 4]
    xbl, ybl, xbs, ybs = [(12, 12, 8, 8), (16, 16, 12, 12), (24, 24, 16, 16), (8, 8, 8, 8), (16, 12, 12, 8)][
        trial % 5]
    xsb, ysb = (w + 4 * xbs - 1) // (4 * xbs), (h + 4 * ybs - 1) // (4 * ybs)
    bp = BlockParams(prec, xbl, ybl, xbs, ybs, xsb, ysb)
    nb = (4 * ysb, 4 * xsb)
    a = {"mv1": rng.integers(-80 << prec, 80 << prec, size=nb + (2,)).astype(np.int16),
         "mv2": rng.integers(-80 << prec, 80 << prec, size=nb + (2,)).astype(np.int16),
         "mode": rng.integers(0, 4, size=nb).astype(np.uint8),
         "dc": rng.integers(-128, 128, size=(3,) + nb).astype(np.int16),
         "split": rng.integers(0, 3, size=(ysb, xsb)).astype(np.uint8)}
    xs, ys = chroma_shift(cf)
    mk = lambda: [rng.integers(-128, 128, size=(h, w)).astype(np.int16)] + [
        rng.integers(-128, 128, size=(h >> ys, w >> xs)).astype(np.int16) for _ in range(2)]
    pic, r1, r2 = mk(), mk(), mk()
    for aos in (0, 1):
        want = oracle.motion_compensate(aos, cf, pic, r1, r2, bp, a["mv1"], a["mv2"], a["mode"], a["dc"], a["split"])
        got = gpu_mc(gpu, aos, cf, bp, a, pic, r1, r2)
        for c in range(3):
            np.testing.assert_array_equal(got[c], want[c], err_msg=f"aos {aos} comp {c}")


@pytest.mark.parametrize("trial", range(8))
def test_weighted_mc_vs_oracle(gpu, oracle, trial):
    """Custom reference picture weights (dgpu_motion_compensate_weighted) against the oracle,
    every prediction mode and chroma format, up to 1080p, 10-bit-range samples (so that large
    weights wrap the reference's int16 block values)."""
    from oracle import BlockParams, chroma_shift
    from test_oracle import MC_WEIGHTS

    rng = np.random.default_rng(700 + trial)
    weights = MC_WEIGHTS[trial % len(MC_WEIGHTS)]
    cf, prec = trial % 3, (trial + 2) % 4
    w, h = [(352, 288), (1920, 1080), (176, 144), (130, 98)][trial % 4]
    xbl, ybl, xbs, ybs = [(12, 12, 8, 8), (16, 16, 12, 12), (8, 8, 8, 8), (16, 12, 12, 8)][trial % 4]
    xsb, ysb = (w + 4 * xbs - 1) // (4 * xbs), (h + 4 * ybs - 1) // (4 * ybs)
    bp = BlockParams(prec, xbl, ybl, xbs, ybs, xsb, ysb)
    nb = (4 * ysb, 4 * xsb)
    a = {"mv1": rng.integers(-60 << prec, 60 << prec, size=nb + (2,)).astype(np.int16),
         "mv2": rng.integers(-60 << prec, 60 << prec, size=nb + (2,)).astype(np.int16),
         "mode": rng.integers(0, 4, size=nb).astype(np.uint8),
         "dc": rng.integers(-512, 512, size=(3,) + nb).astype(np.int16),
         "split": rng.integers(0, 3, size=(ysb, xsb)).astype(np.uint8), "weights": weights}
    xs, ys = chroma_shift(cf)
    mk = lambda: [rng.integers(-512, 512, size=(h, w)).astype(np.int16)] + [
        rng.integers(-512, 512, size=(h >> ys, w >> xs)).astype(np.int16) for _ in range(2)]
    pic, r1, r2 = mk(), mk(), mk()
    for aos in (0, 1):
        want = oracle.motion_compensate(aos, cf, pic, r1, r2, bp, a["mv1"], a["mv2"], a["mode"], a["dc"],
                                        a["split"], 10, 10, weights)
        got = gpu_mc(gpu, aos, cf, bp, a, pic, r1, r2, lbd=10)
        for c in range(3):
            np.testing.assert_array_equal(got[c], want[c], err_msg=f"weights {weights} aos {aos} comp {c}")


def test_weighted_mc_rejects_bad_precision():
    from dirac_b200 import _lib

    lib = _lib.load()
    assert lib.dgpu_motion_compensate_weighted(0, 2, 64, 64, None, None, None, None, None, None, None, None,
                                               None, None, 0, 0, 1, 1, 1, None) == -1


@pytest.mark.parametrize("prec", range(4))
@pytest.mark.parametrize("mode", [1, 2, 3, 0])
def test_add_then_subtract_is_identity(gpu, prec, mode):
    """unit_tests/motion_comp_test.cpp:101-460 (CIF, OLB 12/12/8/8, MV (5,5) and (0,0), each
    precision, REF1 / REF2 / REF1AND2 / intra): ADD then SUBTRACT restores the picture."""
    from oracle import BlockParams

    rng = np.random.default_rng(prec * 7 + mode)
    w, h = 352, 288
    bp = BlockParams(prec, 12, 12, 8, 8, w // 32, h // 32)
    nb = (4 * (h // 32), 4 * (w // 32))
    for mvv in (0, 5):
        a = {"mv1": np.full(nb + (2,), mvv, np.int16), "mv2": np.full(nb + (2,), -mvv, np.int16),
             "mode": np.full(nb, mode, np.uint8), "dc": rng.integers(-100, 100, size=(3,) + nb).astype(np.int16),
             "split": np.full((h // 32, w // 32), 2, np.uint8)}
        pic = [rng.integers(-128, 128, size=s).astype(np.int16) for s in [(h, w), (h // 2, w // 2), (h // 2, w // 2)]]
        r1 = [rng.integers(-128, 128, size=p.shape).astype(np.int16) for p in pic]
        r2 = [rng.integers(-128, 128, size=p.shape).astype(np.int16) for p in pic]
        added = gpu_mc(gpu, 0, 2, bp, a, pic, r1, r2)
        back = gpu_mc(gpu, 1, 2, bp, a, added, r1, r2)
        for c in range(3):
            np.testing.assert_array_equal(back[c], pic[c])


def test_mc_add_with_fused_clip(gpu, oracle):
    from oracle import BlockParams

    rng = np.random.default_rng(8)
    w, h = 176, 144
    bp = BlockParams(2, 12, 12, 8, 8, w // 32 + 1, h // 32 + 1)
    nb = (4 * bp.ynum_sb, 4 * bp.xnum_sb)
    a = {"mv1": rng.integers(-30, 30, size=nb + (2,)).astype(np.int16),
         "mv2": rng.integers(-30, 30, size=nb + (2,)).astype(np.int16),
         "mode": rng.integers(0, 4, size=nb).astype(np.uint8),
         "dc": rng.integers(-128, 128, size=(3,) + nb).astype(np.int16),
         "split": rng.integers(0, 3, size=(bp.ynum_sb, bp.xnum_sb)).astype(np.uint8)}
    pic = [rng.integers(-200, 200, size=s).astype(np.int16) for s in [(h, w), (h // 2, w // 2), (h // 2, w // 2)]]
    r1 = [rng.integers(-128, 128, size=p.shape).astype(np.int16) for p in pic]
    want = oracle.motion_compensate(0, 2, pic, r1, r1, bp, a["mv1"], a["mv2"], a["mode"], a["dc"], a["split"])
    for x in want:
        oracle.clip(x, 8)
    got = gpu_mc(gpu, 0, 2, bp, a, pic, r1, r1, clip=(8, 8))
    for c in range(3):
        np.testing.assert_array_equal(got[c], want[c])
