"""The heterogeneous picture batch (dgpu_batch_*) against the oracle's restatement of the
encoder's per-picture coding: pictures of different sizes, chroma formats, bit depths,
filters, depths, block parameters and precisions, intra and inter (one and two references,
P and B lambdas), coded in one batch, each equal bit for bit to its own coding (reconstructed
pictures, coefficients, quantised indices, band choices, code-block skips), on a first run
(tuning and graph capture) and a replayed second run."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bp(w, h, prec, xblen, yblen, xbsep, ybsep):
    from dirac_b200._lib import BlockParams

    return BlockParams(precision=prec, xblen=xblen, yblen=yblen, xbsep=xbsep, ybsep=ybsep,
                       xnum_sb=(w + 4 * xbsep - 1) // (4 * xbsep), ynum_sb=(h + 4 * ybsep - 1) // (4 * ybsep))


# (w, h, chroma, depth bits, filter, wlt depth, refs (0 intra), is_b, qf, (prec, xblen, yblen, xbsep, ybsep))
CASES = [
    (176, 144, "420", 8, 1, 3, 0, 0, 7.0, None),
    (176, 144, "420", 8, 0, 3, 1, 0, 7.0, (2, 12, 12, 8, 8)),
    (192, 128, "422", 10, 2, 4, 2, 1, 6.0, (3, 16, 16, 12, 12)),
    (160, 96, "444", 12, 4, 4, 0, 0, 8.0, None),
    (176, 144, "420", 8, 5, 5, 2, 0, 7.5, (2, 16, 16, 12, 12)),
    (128, 128, "420", 8, 3, 3, 1, 0, 5.0, (1, 12, 12, 8, 8)),
]
CFORMAT = {"444": 0, "422": 1, "420": 2}


def build_inputs():
    import torch

    from dirac_b200 import synth
    from dirac_b200.motion import MotionEstimator

    pics, motion, planes, refs_np, me_np, params = [], [], [], [], [], []
    for i, (w, h, chroma, bits, filt, depth, nref, is_b, qf, blk) in enumerate(CASES):
        seq = synth.make_sequence(w, h, 3, n_rects=4, vmax=4, seed=300 + i, bit_depth=bits, chroma=chroma)
        frames = [[synth.to_signed(p, bits) for p in f] for f in seq]
        cur = frames[1]
        prm = dict(cformat=CFORMAT[chroma], width=w, height=h, luma_depth=bits, chroma_depth=bits, filter=filt,
                   wlt_depth=depth, intra=int(nref == 0), is_b=is_b, qf=qf, cpd=20.0, intra_ratio=0.0)
        m = None
        rp = None
        me = None
        if nref:
            prec, xbl, ybl, xbs, ybs = blk
            bp = _bp(w, h, prec, xbl, ybl, xbs, ybs)
            prm["bp"] = bp
            prm.update(mv_precision=prec, xblen=xbl, yblen=ybl, xbsep=xbs, ybsep=ybs)
            rp = [frames[0]] if nref == 1 else [frames[0], frames[2]]
            dev = [[torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in f] for f in [cur] + rp]
            est = MotionEstimator(bp, CFORMAT[chroma], bits).Estimate(dev[0], dev[1], dev[2] if nref == 2 else None,
                                                                       lambda_=10.0)
            nb = est["mode"].numel()
            prm["intra_ratio"] = float((est["mode"] == 0).sum().item()) / nb
            m = {"ref1": dev[1], "ref2": dev[2] if nref == 2 else None, "mv1": est["mv"][0].contiguous(),
                 "mv2": est["mv"][1].contiguous() if nref == 2 else None, "mode": est["mode"], "dc": est["dc"],
                 "split": est["split"]}
            me = {"mv": [t.cpu().numpy() for t in est["mv"]], "mode": est["mode"].cpu().numpy(),
                  "dc": est["dc"].cpu().numpy(), "split": est["split"].cpu().numpy()}
        pics.append(prm)
        motion.append(m)
        planes.append(cur)
        refs_np.append(rp)
        me_np.append(me)
        params.append(prm)
    return pics, motion, planes, refs_np, me_np


def load_planes(batch, planes):
    for k, pl in enumerate(planes):
        batch.load(k, pl)


def test_picture_batch_matches_oracle(gpu, oracle):
    import torch

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
    from oracle_encoder import code_picture

    from dirac_b200 import quant
    from dirac_b200.batch import BANDS, CBSKIP, COEFF, QINDEX, RECON, PictureBatch

    pics, motion, planes, refs, me = build_inputs()
    want = [code_picture(p, pl, quant.band_weights, quant.code_blocks, oracle, refs=r, me=m)
            for p, pl, r, m in zip(pics, planes, refs, me)]
    batch = PictureBatch(pics, motion)
    for run in range(2):
        load_planes(batch, planes)
        batch.run()
        torch.cuda.synchronize()
        for k, (data, res) in enumerate(want):
            msg = f"run {run} picture {k}"
            nb = 3 * pics[k]["wlt_depth"] + 1
            for c in range(3):
                cm = f"{msg} component {c}"
                np.testing.assert_array_equal(batch.read(k, RECON, c), data[c].ravel(), err_msg=cm)
                np.testing.assert_array_equal(batch.read(k, COEFF, c), res["coeff"][c].ravel(), err_msg=cm)
                np.testing.assert_array_equal(batch.read(k, QINDEX, c), res["qindex"][c].ravel(), err_msg=cm)
                b = batch.read(k, BANDS, c).reshape(nb, 3)
                sk = res["skip"][c]
                np.testing.assert_array_equal(b[:, 1], sk, err_msg=cm)
                np.testing.assert_array_equal(b[:, 0][sk == 0], res["qidx"][c][sk == 0], err_msg=cm)
                np.testing.assert_array_equal(b[:, 2], res["bits"][c], err_msg=cm)
                np.testing.assert_array_equal(batch.read(k, CBSKIP, c), res["cb_skip"][c], err_msg=cm)
    batch.close()


# Filters and transform depths given to the full-size pictures in turn, so that every filter of
# the heterogeneous workload (both Haar shifts, LeGall (5,3), Deslauriers-Dubuc (13,7), Fidelity,
# Daubechies (9,7)) and every depth (3-5) occurs at the workload's real sizes.
FULL_SIZE_FILTERS = [3, 1, 2, 5, 6, 4, 6, 2]
FULL_SIZE_DEPTHS = [3, 4, 5, 3, 4, 5, 5, 4]


def test_heterogeneous_workload_at_full_size_matches_oracle(gpu, oracle):
    """The bench's heterogeneous batch at its real picture sizes: two pictures (one P, one B) of
    each class -- 352x288 4:2:0 8-bit, 720x576 4:2:0 8-bit, 1280x720 4:2:0 10-bit, 1920x1080
    4:2:2 10-bit -- with motion from the library's estimation, coded in one batch; every picture
    equal bit for bit to the oracle's coding of it alone, on a first and a replayed run."""
    import torch

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
    from oracle_encoder import code_picture

    from dirac_b200 import hetero as H
    from dirac_b200 import quant
    from dirac_b200.batch import BANDS, CBSKIP, QINDEX, RECON, PictureBatch

    pictures, motion, planes, keep = H.make_inputs(per_class=2, seed=5)
    for k, p in enumerate(pictures):
        p["filter"], p["wlt_depth"] = FULL_SIZE_FILTERS[k], FULL_SIZE_DEPTHS[k]
    assert [(p["width"], p["height"], p["cformat"], p["luma_depth"]) for p in pictures[::2]] == \
        [(352, 288, 2, 8), (720, 576, 2, 8), (1280, 720, 2, 10), (1920, 1080, 1, 10)]
    want = []
    for p, m, pl in zip(pictures, motion, planes):
        bp = p["bp"]
        op = dict(p, mv_precision=bp.precision, xblen=bp.xblen, yblen=bp.yblen, xbsep=bp.xbsep, ybsep=bp.ybsep)
        refs = [[t.cpu().numpy() for t in m["ref1"]]]
        mvs = [m["mv1"].cpu().numpy()]
        if m["ref2"] is not None:
            refs.append([t.cpu().numpy() for t in m["ref2"]])
            mvs.append(m["mv2"].cpu().numpy())
        me = {"mv": mvs, "mode": m["mode"].cpu().numpy(), "dc": m["dc"].cpu().numpy(),
              "split": m["split"].cpu().numpy()}
        want.append(code_picture(op, [t.cpu().numpy() for t in pl], quant.band_weights, quant.code_blocks, oracle,
                                 refs=refs, me=me))
    batch = PictureBatch(pictures, motion)
    for run in range(2):
        load_planes(batch, planes)
        batch.run()
        torch.cuda.synchronize()
        for k, (data, res) in enumerate(want):
            msg = f"run {run} picture {k}"
            nb = 3 * pictures[k]["wlt_depth"] + 1
            for c in range(3):
                cm = f"{msg} component {c}"
                np.testing.assert_array_equal(batch.read(k, RECON, c), data[c].ravel(), err_msg=cm)
                np.testing.assert_array_equal(batch.read(k, QINDEX, c), res["qindex"][c].ravel(), err_msg=cm)
                b = batch.read(k, BANDS, c).reshape(nb, 3)
                sk = res["skip"][c]
                np.testing.assert_array_equal(b[:, 1], sk, err_msg=cm)
                np.testing.assert_array_equal(b[:, 0][sk == 0], res["qidx"][c][sk == 0], err_msg=cm)
                np.testing.assert_array_equal(batch.read(k, CBSKIP, c), res["cb_skip"][c], err_msg=cm)
    batch.close()
    del keep
