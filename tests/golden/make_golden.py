"""Generate the golden fixtures in this directory by running the reference codec itself.

Needs oracle/_ref/libdirac_ref.so (the reference's own C++, plain-C build, compiled from
its sources by `make -C oracle`).  Inputs are seeded, so re-running reproduces the files.

    python tests/golden/make_golden.py [dwt convert mc me quant encode decode adaptive bands prefilter hd1080 uhd
                                        fields]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
from oracle import Reference  # noqa: E402


def dwt_cases(ref):
    rng = np.random.default_rng(20261203)
    out = {}
    # (w, h, depth): odd padding on both axes; level sides stay >= 6
    shapes = [(70, 38, 3), (45, 52, 2), (64, 48, 4)]
    for filt in range(7):
        for k, (w, h, depth) in enumerate(shapes):
            mul = 1 << depth
            cw, ch = (w + mul - 1) // mul * mul, (h + mul - 1) // mul * mul
            pic = rng.integers(-128, 128, size=(h, w)).astype(np.int16)
            coeff = ref.dwt_forward(filt, depth, pic, cw, ch)
            noisy = (coeff + rng.integers(-9, 10, size=coeff.shape)).astype(np.int32)
            back = ref.dwt_backward(filt, depth, noisy, w, h)
            key = f"f{filt}_c{k}"
            out[key + "_pic"] = pic
            out[key + "_coeff"] = coeff
            out[key + "_noisy"] = noisy
            out[key + "_back"] = back
            out[key + "_meta"] = np.array([filt, depth, w, h, cw, ch], np.int32)
    return out


def conv_cases(ref):
    rng = np.random.default_rng(7)
    out = {}
    for k, (w, h, bd) in enumerate([(40, 24, 8), (33, 17, 10), (8, 8, 8)]):
        pic = rng.integers(-(1 << (bd - 1)), 1 << (bd - 1), size=(h, w)).astype(np.int16)
        out[f"up{k}_pic"] = pic
        out[f"up{k}_out"] = ref.upconvert(pic, bd)
        out[f"up{k}_meta"] = np.array([w, h, bd], np.int32)
    for k, (w, h) in enumerate([(64, 50), (49, 31), (24, 24)]):
        pic = rng.integers(-128, 128, size=(h, w)).astype(np.int16)
        out[f"down{k}_pic"] = pic
        out[f"down{k}_out"] = ref.downconvert(pic)
    return out


def mc_cases(ref):
    """OBMC of small pictures: (w, h, cformat, precision, olb, nref) with random vectors,
    modes, DC values and superblock splits, for ADD and SUBTRACT."""
    from oracle import BlockParams, chroma_shift

    rng = np.random.default_rng(42)
    out = {}
    cases = [(96, 64, 2, 2, (12, 12, 8, 8), 2), (100, 72, 1, 3, (16, 16, 12, 12), 2),
             (64, 48, 0, 1, (8, 8, 8, 8), 1), (72, 56, 2, 0, (16, 12, 12, 8), 2)]
    # then custom reference picture weights (ref1, ref2, precision bits) on 10-bit-range samples
    cases += [(96, 64, 2, 2, (12, 12, 8, 8), 2, (3, 5, 3)), (72, 56, 1, 1, (16, 16, 12, 12), 2, (-2, 7, 2)),
              (64, 48, 0, 3, (8, 8, 8, 8), 1, (1, 1, 0)), (80, 48, 2, 2, (16, 12, 12, 8), 2, (255, 1, 8))]
    for k, case in enumerate(cases):
        w, h, cf, prec, olb, nref = case[:6]
        wts = case[6] if len(case) > 6 else (1, 1, 1)
        amp = 128 if len(case) == 6 else 512
        xbl, ybl, xbs, ybs = olb
        xsb, ysb = (w + 4 * xbs - 1) // (4 * xbs), (h + 4 * ybs - 1) // (4 * ybs)
        nb = (4 * ysb, 4 * xsb)
        rr = 24 << prec
        mv1 = rng.integers(-rr, rr, size=nb + (2,)).astype(np.int16)
        mv2 = rng.integers(-rr, rr, size=nb + (2,)).astype(np.int16)
        mode = rng.integers(0, 4 if nref == 2 else 2, size=nb).astype(np.uint8)
        dc = rng.integers(-amp, amp, size=(3,) + nb).astype(np.int16)
        split = rng.integers(0, 3, size=(ysb, xsb)).astype(np.uint8)
        xs, ys = chroma_shift(cf)

        def mk():
            return [rng.integers(-amp, amp, size=(h, w)).astype(np.int16)] + \
                   [rng.integers(-amp, amp, size=(h >> ys, w >> xs)).astype(np.int16) for _ in range(2)]

        pic, r1, r2 = mk(), mk(), mk()
        bp = BlockParams(prec, xbl, ybl, xbs, ybs, xsb, ysb)
        key = f"mc{k}"
        out[key + "_meta"] = np.array([w, h, cf, prec, xbl, ybl, xbs, ybs, xsb, ysb, nref], np.int32)
        out[key + "_wt"] = np.array(wts, np.int32)
        for name, a in (("mv1", mv1), ("mv2", mv2), ("mode", mode), ("dc", dc), ("split", split)):
            out[f"{key}_{name}"] = a
        for c in range(3):
            out[f"{key}_pic{c}"] = pic[c]
            out[f"{key}_r1_{c}"] = r1[c]
            out[f"{key}_r2_{c}"] = r2[c]
        for aos in (0, 1):
            bd = 8 if amp == 128 else 10
            res = ref.motion_compensate(aos, cf, pic, r1, r2 if nref == 2 else None, bp, mv1, mv2, mode, dc,
                                        split, bd, bd, wts)
            for c in range(3):
                out[f"{key}_out{aos}_{c}"] = res[c]
    return out


def me_cases(ref):
    """Motion estimation (pel pyramid, sub-pel, mode decision) of small synthetic pictures."""
    sys.path.insert(0, os.path.join(HERE, "..", "..", "dirac-research_b200"))
    from dirac_b200 import synth
    from oracle import BlockParams

    out = {}
    cases = [(176, 144, (12, 12, 8, 8), 2, 2, "420", 3), (160, 128, (16, 16, 12, 12), 3, 2, "422", 4),
             (192, 144, (8, 8, 8, 8), 1, 1, "420", 5)]
    for k, (w, h, olb, prec, nref, chroma, seed) in enumerate(cases):
        seq = synth.make_sequence(w, h, 3, n_rects=6, vmax=6, seed=seed, chroma=chroma)
        f = [[synth.to_signed(p) for p in fr] for fr in seq]
        xbl, ybl, xbs, ybs = olb
        bp = BlockParams(prec, xbl, ybl, xbs, ybs, (w + 4 * xbs - 1) // (4 * xbs), (h + 4 * ybs - 1) // (4 * ybs))
        cf = {"444": 0, "422": 1, "420": 2}[chroma]
        lam = 9.0 + k
        res = ref.motion_estimate(cf, f[1], f[0], f[2] if nref == 2 else None, bp, lam, 3)
        key = f"me{k}"
        out[key + "_meta"] = np.array([w, h, cf, prec, xbl, ybl, xbs, ybs, bp.xnum_sb, bp.ynum_sb, nref], np.int32)
        out[key + "_lambda"] = np.array([lam], np.float32)
        for c in range(3):
            out[f"{key}_pic{c}"] = f[1][c]
            out[f"{key}_r1_{c}"] = f[0][c]
            out[f"{key}_r2_{c}"] = f[2][c]
        for name, a in res.items():
            out[f"{key}_{name}"] = a
    return out


def quant_cases(ref):
    """Residue coding (quantiser choice, quantisation, reconstruction) of transformed
    synthetic components, intra and inter, run by the reference's own classes."""
    sys.path.insert(0, os.path.join(HERE, "..", "..", "dirac-research_b200"))
    from dirac_b200 import synth
    from oracle import Oracle

    orc = Oracle()
    out = {}
    cases = [(176, 144, 4, 6, 1, 0, 7), (176, 144, 4, 0, 0, 1, 7), (128, 96, 3, 1, 1, 2, 5),
             (160, 128, 4, 2, 0, 0, 9)]
    for k, (w, h, depth, filt, intra, comp, qf) in enumerate(cases):
        seq = synth.make_sequence(w, h, 2, n_rects=6, vmax=6, seed=70 + k)
        f = [synth.to_signed(p) for p in seq[0]]
        g = [synth.to_signed(p) for p in seq[1]]
        pic = f[comp] if intra else np.clip(f[comp].astype(np.int32) - g[comp], -128, 127).astype(np.int16)
        coeff = orc.dwt_forward(filt, depth, pic)
        lam = 10 ** ((12 - qf) / 2.5) / 16 * (1 if intra else 4)
        r = ref.code_residue(2, w, h, comp, intra, filt, depth, coeff, lam)
        key = f"q{k}"
        out[key + "_meta"] = np.array([w, h, depth, filt, intra, comp], np.int32)
        out[key + "_lambda"] = np.array([lam], np.float32)
        out[key + "_coeff"] = coeff
        for name, a in r.items():
            out[f"{key}_{name}"] = a
    return out


ENCODE_CASES = [
    # (name, w, h, frames, seed A, seed B, switch frame or None, n_rects, vmax, qf, num_l1,
    #  intra filter, inter filter, depth, xblen, yblen, xbsep, ybsep, precision)
    ("cif", 352, 288, 16, 1, None, None, 8, 8, 7.0, 19, 1, 0, 4, 12, 12, 8, 8, 2),
    ("reconfig", 176, 144, 14, 11, 12, 3, 4, 4, 7.0, 19, 1, 0, 3, 12, 12, 8, 8, 2),
    ("cut_b", 176, 144, 14, 11, 12, 5, 4, 4, 7.0, 19, 1, 0, 3, 12, 12, 8, 8, 2),
    ("cut_p", 176, 144, 14, 11, 12, 7, 4, 4, 7.0, 19, 1, 0, 3, 12, 12, 8, 8, 2),
    ("gop", 176, 144, 13, 21, None, None, 6, 6, 5.0, 2, 6, 2, 4, 16, 16, 12, 12, 3),
]


def encode_inputs(case):
    """8-bit frames of one ENCODE_CASES entry and its RefEncParams fields."""
    sys.path.insert(0, os.path.join(HERE, "..", "..", "dirac-research_b200"))
    from dirac_b200 import synth

    (name, w, h, n, sa, sb, sw, nr, vm, qf, nl1, fi, fr, depth, xbl, ybl, xbs, ybs, prec) = case
    seq = synth.make_sequence(w, h, n, n_rects=nr, vmax=vm, seed=sa)
    if sb is not None:
        seq = seq[:sw] + synth.make_sequence(w, h, n, n_rects=nr, vmax=vm, seed=sb)[sw:]
    cfg = dict(video_format=0, cformat=2, width=w, height=h, qf=qf, l1_sep=3, num_l1=nl1, cpd=20.0, xblen=xbl,
               yblen=ybl, xbsep=xbs, ybsep=ybs, mv_precision=prec, intra_filter=fi, inter_filter=fr, wlt_depth=depth)
    return seq, cfg


# The 1080p coding workload the bench times: 1920x1080 4:2:0 8-bit, 24 rectangles moving at up to
# 24 px/frame, the HD1080P50 preset (L1 separation 3, 7 L1 pictures per GOP), QF 7, DAUB9_7 intra /
# DD9_7 inter depth 4, OBMC 16x16 at separation 12, quarter-pel motion vectors.  The fixture codes
# the first HD_FRAMES frames of the bench's 32-frame sequence (seed 1000) as one sequence, as the
# bench's CPU baseline does.
HD_PARAMS = dict(video_format=14, cformat=2, width=1920, height=1080, qf=7.0, l1_sep=3, num_l1=7, cpd=32.0,
                 xblen=16, yblen=16, xbsep=12, ybsep=12, mv_precision=2, intra_filter=6, inter_filter=0,
                 wlt_depth=4)
HD_FRAMES = 10
HD_SEQUENCE_FRAMES = 32
HD_SEED = 1000


def hd_inputs():
    """8-bit frames of the 1080p case and its RefEncParams fields."""
    sys.path.insert(0, os.path.join(HERE, "..", "..", "dirac-research_b200"))
    from dirac_b200 import synth

    seq = synth.make_sequence(1920, 1080, HD_SEQUENCE_FRAMES, n_rects=24, vmax=24, seed=HD_SEED, bit_depth=8,
                              chroma="420")
    return seq[:HD_FRAMES], dict(HD_PARAMS)


def hd_cases():
    """The reference encoder on the 1080p case through its public API, with the initial
    entropy-correction factors kept (frozen) and as it ships (adaptive), arithmetic coding:
    CRC-32 of every locally decoded plane, the picture types and the bitstream's length and
    CRC-32; and the reference decoder's CRC-32s of that bitstream decoded."""
    import zlib

    from oracle import reference_decode, reference_encode_stream

    seq, cfg = hd_inputs()
    out = {}
    for tag, freeze in (("frozen", True), ("adaptive", False)):
        rec, ptype, stream = reference_encode_stream(cfg, seq, freeze=freeze)
        out[tag + "_crc"] = np.array([[zlib.crc32(np.ascontiguousarray(p).tobytes()) for p in f] for f in rec],
                                     np.uint32)
        out[tag + "_ptype"] = ptype
        out[tag + "_stream_bytes"] = np.array(len(stream), np.int64)
        out[tag + "_stream_crc"] = np.array(zlib.crc32(bytes(stream)), np.uint32)
        dec = reference_decode(stream, cfg["width"], cfg["height"], cfg["cformat"], len(seq))
        if any(f is None for f in dec):
            raise RuntimeError("hd1080: the reference decoder did not deliver every frame")
        out[tag + "_decode_crc"] = np.array([[zlib.crc32(np.ascontiguousarray(p).tobytes()) for p in f]
                                             for f in dec], np.uint32)
    return out


# The 3840x2160 4:2:2 10-bit workload: 48 rectangles moving at up to 64 px/frame, Deslauriers-Dubuc
# (9,7) depth 5, OBMC 16x16 at separation 12, quarter-pel vectors, motion estimation over the
# reference's pyramid of depth 7 (pixel_match.cpp:94-95 at this size).  Frame 1 is a B picture
# between frames 0 and 2.
UHD_SIZE = (3840, 2160)
UHD_SEED = 2160
UHD_LAMBDA = 10.0


def uhd_inputs():
    """Three 10-bit 4:2:2 frames as int16 codec samples, and the block parameters."""
    sys.path.insert(0, os.path.join(HERE, "..", "..", "dirac-research_b200"))
    from dirac_b200 import synth
    from oracle import BlockParams

    w, h = UHD_SIZE
    seq = synth.make_sequence(w, h, 3, n_rects=48, vmax=64, seed=UHD_SEED, bit_depth=10, chroma="422")
    frames = [[synth.to_signed(p, 10) for p in fr] for fr in seq]
    bp = BlockParams(2, 16, 16, 12, 12, (w + 47) // 48, (h + 47) // 48)
    return frames, bp


def crc(a):
    import zlib

    return zlib.crc32(np.ascontiguousarray(a).tobytes())


def uhd_cases(ref):
    """The reference's stages on the 4K workload (CRC-32s, the arrays being tens of MB): motion
    estimation of the B picture (stages 1-3), OBMC SUBTRACT and ADD with those motion data,
    upconversion of a reference, and forward and inverse DD9_7 depth-5 transforms of each
    component of the B picture."""
    f, bp = uhd_inputs()
    out = {}
    me = ref.motion_estimate(1, f[1], f[0], f[2], bp, UHD_LAMBDA, 3, luma_depth=10)
    for k, v in me.items():
        out["me_" + k] = np.array(crc(v), np.uint32)
    nref = me["mv"].shape[0]
    mv1, mv2 = me["mv"][0], me["mv"][1 if nref > 1 else 0]
    for aos in (0, 1):
        res = ref.motion_compensate(aos, 1, f[1], f[0], f[2], bp, mv1, mv2, me["mode"], me["dc"], me["split"],
                                    luma_depth=10, chroma_depth=10)
        out[f"mc{aos}"] = np.array([crc(c) for c in res], np.uint32)
    out["up"] = np.array([crc(ref.upconvert(c, 10)) for c in f[0]], np.uint32)
    fwd, back = [], []
    for c in range(3):
        pic = f[1][c]
        co = ref.dwt_forward(0, 5, pic)
        fwd.append(crc(co))
        back.append(crc(ref.dwt_backward(0, 5, co, pic.shape[1], pic.shape[0])))
    out["dwt_fwd"] = np.array(fwd, np.uint32)
    out["dwt_back"] = np.array(back, np.uint32)
    out["in"] = np.array([[crc(c) for c in fr] for fr in f], np.uint32)
    return out


def encode_cases():
    """The reference encoder run through its public API (initial entropy-correction factors
    kept, as a coding loop without the arithmetic coder does): CRC-32 of every locally
    decoded plane and the picture types, for sequences that exercise the plain GOP, the
    switch to P-only sub-groups and cut detection."""
    import zlib

    from oracle import reference_encode

    out = {}
    for case in ENCODE_CASES:
        seq, cfg = encode_inputs(case)
        rec, ptype, nbytes = reference_encode(cfg, seq, freeze=True)
        name = case[0]
        out[name + "_crc"] = np.array([[zlib.crc32(np.ascontiguousarray(p).tobytes()) for p in f] for f in rec],
                                      np.uint32)
        out[name + "_ptype"] = ptype
    return out


# Field coding (FieldSequenceCompressor): (name, w, h, frames, seed A, seed B, switch frame or
# None, n_rects, vmax, qf, num_l1, intra filter, inter filter, depth, xblen, yblen, xbsep, ybsep,
# precision, video format).  The CIF preset puts the top field first, the custom one (0) the
# bottom field; the third sequence switches content to trigger cut detection and the switch to
# P-only sub-groups on fields.
FIELD_CASES = [
    ("field_cif_tff", 352, 288, 8, 31, None, None, 8, 8, 7.0, 19, 1, 0, 4, 12, 12, 8, 8, 2, 4),
    ("field_bff", 176, 144, 10, 32, None, None, 6, 6, 5.0, 2, 6, 2, 3, 16, 16, 12, 12, 3, 0),
    ("field_cut", 176, 144, 12, 41, 42, 5, 4, 4, 7.0, 19, 1, 0, 3, 12, 12, 8, 8, 2, 0),
]


# top field first as the reference's video-format presets set it (video_format_defaults.cpp:
# true by default, false for the custom and 525-line formats)
TOP_FIELD_FIRST = {0: 0, 4: 1}


def field_inputs(case):
    """8-bit frames of one FIELD_CASES entry and its RefEncParams fields (field coding)."""
    seq, cfg = encode_inputs(case[:19])
    cfg.update(video_format=case[19], field_coding=1)
    return seq, cfg


def field_cases():
    """The reference encoder in field-coding mode through its public API: CRC-32 of every
    locally decoded field's planes it returns (all but the last frame's two) and the types it
    reports (-2 for first fields, -1 for fields not returned), with the initial
    entropy-correction factors kept and with the stock adaptive ones."""
    import zlib

    from oracle import reference_encode

    out = {}
    for case in FIELD_CASES:
        seq, cfg = field_inputs(case)
        for tag, freeze in (("", True), ("_adaptive", False)):
            rec, ptype, _ = reference_encode(cfg, seq, freeze=freeze)
            # the encoder's API shows every frame but the sequence's last: its fields stay -1
            if (ptype[:-2] == -1).any():
                raise RuntimeError(f"{case[0]}: a field was never returned")
            out[case[0] + tag + "_crc"] = np.array(
                [[zlib.crc32(np.ascontiguousarray(p).tobytes()) for p in f] for f in rec], np.uint32)
            out[case[0] + tag + "_ptype"] = ptype
    return out


def decode_cases():
    """The reference decoder run through its public API on the reference encoder's bitstream
    of each ENCODE_CASES sequence: CRC-32 of every decoded plane by frame number, and the
    stream length."""
    import zlib

    from oracle import reference_decode, reference_encode_stream

    out = {}
    for case in ENCODE_CASES:
        seq, cfg = encode_inputs(case)
        _, _, stream = reference_encode_stream(cfg, seq, freeze=True)
        dec = reference_decode(stream, cfg["width"], cfg["height"], cfg["cformat"], len(seq))
        if any(f is None for f in dec):
            raise RuntimeError(f"{case[0]}: the reference decoder did not deliver every frame")
        name = case[0]
        out[name + "_crc"] = np.array([[zlib.crc32(np.ascontiguousarray(p).tobytes()) for p in f] for f in dec],
                                      np.uint32)
        out[name + "_bytes"] = np.array(len(stream), np.int64)
    return out


def adaptive_cases():
    """The stock reference encoder (entropy-correction factors adapted from its coder's byte
    counts, as it ships) on each ENCODE_CASES sequence, with arithmetic coding and with
    variable-length coding (-use_vlc, "<name>_vlc_*"): CRC-32 of every locally decoded plane,
    the picture types, and the bitstream's length and CRC-32."""
    import zlib

    from oracle import reference_encode_stream

    out = {}
    for case in ENCODE_CASES:
        seq, cfg = encode_inputs(case)
        name = case[0]
        for tag, vlc in (("", 0), ("_vlc", 1)):
            rec, ptype, stream = reference_encode_stream(dict(cfg, use_vlc=vlc), seq, freeze=False)
            out[name + tag + "_crc"] = np.array([[zlib.crc32(np.ascontiguousarray(p).tobytes()) for p in f]
                                                 for f in rec], np.uint32)
            out[name + tag + "_ptype"] = ptype
            out[name + tag + "_stream_bytes"] = np.array(len(stream), np.int64)
            out[name + tag + "_stream_crc"] = np.array(zlib.crc32(bytes(stream)), np.uint32)
    return out


def band_cases(ref):
    """The reference's band coders on seeded components (intra and inter, several filters,
    depths and sizes), arithmetic and variable-length (-use_vlc): the quantiser choices and the
    CRC-32 and length of every coded band's data, with the inputs to rebuild them (seed, size,
    filter, depth, lambda)."""
    import zlib

    out = {}
    for k, (intra, filt, depth, w, h, lam) in enumerate(BAND_CASES):
        rng = np.random.default_rng(900 + k)
        pic = rng.integers(-60, 60, size=(h, w)).astype(np.int16)
        co = ref.dwt_forward(filt, depth, pic)
        r = ref.code_residue_bytes(2, w, h, 0, intra, filt, depth, co, lam)
        start = 0
        crcs = []
        for b in range(3 * depth + 1, 0, -1):  # coding order, DC band first
            n = int(r["band_bytes"][b - 1])
            crcs.append(zlib.crc32(r["data"][start:start + n].tobytes()))
            start += n
        out[f"c{k}_band_bytes"] = r["band_bytes"]
        out[f"c{k}_band_crc"] = np.array(crcs[::-1], np.uint32)  # band-list order
        out[f"c{k}_qidx"] = r["qidx"]
        out[f"c{k}_skip"] = r["skip"]
        v = ref.code_residue_vlc_bytes(2, w, h, 0, intra, filt, depth, co, lam)
        start, vcrc = 0, []
        for b in range(3 * depth + 1, 0, -1):
            n = int(v["band_bytes"][b - 1])
            vcrc.append(zlib.crc32(v["data"][start:start + n].tobytes()))
            start += n
        out[f"c{k}_vlc_band_bytes"] = v["band_bytes"]
        out[f"c{k}_vlc_band_crc"] = np.array(vcrc[::-1], np.uint32)
        out[f"c{k}_vlc_compress_bytes"] = v["compress_bytes"]
        out[f"c{k}_wt"] = r["wt"]
        out[f"c{k}_ecf"] = r["ecf"]
        out[f"c{k}_ncb"] = r["ncb"]
        out[f"c{k}_cb_skip"] = r["cb_skip"]
    return out


# (width, height, strength) of prefilter_cases
PREFILTER_CASES = [(64, 48, 0), (37, 23, 3), (48, 40, 5), (33, 17, 8), (40, 32, 9), (16, 9, 11)]


# (width, height, quality factor, strength) of the RECTLP cases
RECTLP_CASES = [(48, 40, 7.0, 0), (17, 17, 2.0, 1), (33, 21, 10.0, 5), (64, 24, 0.5, 3), (40, 36, 12.0, 10)]


# (width, height, quality factor, strength) of the DIAGLP cases: filter bandwidth indices 9 down
# to 2 (the last clamped), partial and full blending factors, and one pair that leaves the
# component alone (bandwidth above 0.9)
DIAGLP_CASES = [(48, 40, 3.0, 0), (17, 17, 4.5, 2), (33, 21, 4.5, 3), (7, 7, 5.7, 5), (40, 36, 5.8, 6),
                (29, 35, 6.2, 7), (64, 24, 7.2, 9), (23, 9, 6.0, 10), (31, 13, 7.0, 0)]


def prefilter_cases(ref):
    """CWMFilterComponent, LPFilter (RECTLP) and DiagFilter (DIAGLP) of the reference on seeded
    components."""
    out = {}
    for k, (w, h, strength) in enumerate(PREFILTER_CASES):
        rng = np.random.default_rng(500 + k)
        pic = rng.integers(-128, 128, size=(h, w)).astype(np.int16)
        out[f"c{k}_in"] = pic
        out[f"c{k}_out"] = ref.cwm_filter(pic, strength)
    for k, (w, h, qf, strength) in enumerate(RECTLP_CASES):
        rng = np.random.default_rng(600 + k)
        pic = rng.integers(-300, 300, size=(h, w)).astype(np.int16)
        out[f"lp{k}_in"] = pic
        out[f"lp{k}_out"] = ref.rect_lp_filter(pic, qf, strength)
    for k, (w, h, qf, strength) in enumerate(DIAGLP_CASES):
        rng = np.random.default_rng(700 + k)
        pic = rng.integers(-300, 300, size=(h, w)).astype(np.int16)
        out[f"dg{k}_in"] = pic
        out[f"dg{k}_out"] = ref.diag_lp_filter(pic, qf, strength)
    return out


# (intra, filter, depth, width, height, lambda) of band_cases
BAND_CASES = [(1, 1, 4, 176, 144, 5.0), (0, 0, 4, 176, 144, 30.0), (1, 6, 3, 88, 72, 3.0),
              (0, 2, 5, 352, 288, 100.0), (1, 3, 2, 64, 48, 1.0), (0, 4, 3, 96, 80, 8.0)]


def main(argv=None):
    """Writes the named fixtures (default: all)."""
    names = (argv if argv is not None else sys.argv[1:]) or ["dwt", "convert", "mc", "me", "quant", "encode",
                                                              "decode", "adaptive", "bands", "prefilter",
                                                              "hd1080", "uhd", "fields"]
    ref = Reference()
    makers = {"dwt": lambda: dwt_cases(ref), "convert": lambda: conv_cases(ref), "mc": lambda: mc_cases(ref),
              "me": lambda: me_cases(ref), "quant": lambda: quant_cases(ref), "encode": encode_cases,
              "decode": decode_cases, "adaptive": adaptive_cases, "bands": lambda: band_cases(ref),
              "prefilter": lambda: prefilter_cases(ref), "hd1080": hd_cases,
              "uhd": lambda: uhd_cases(ref), "fields": field_cases}
    for n in names:
        np.savez_compressed(os.path.join(HERE, n + ".npz"), **makers[n]())
    print("wrote " + ", ".join(n + ".npz" for n in names))


if __name__ == "__main__":
    main()
