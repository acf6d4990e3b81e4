"""TEST INFRASTRUCTURE ONLY: the reference decoder's picture decoding restated over the oracle's
stages (oracle/dirac_oracle*.c through oracle.Oracle).

PictureDecompressor::Decompress (libdirac_decoder/picture_decompress.cpp:73-212), from the
point where the picture's coefficients and motion data have been entropy-decoded: per
component the dequantisation (CompDecompressor::Decompress and the band decoders,
comp_decompress.cpp:64-163, band_codec_template.h:204-357, 470-557) and the inverse transform
(WaveletTransform::Transform BACKWARD), or zero samples when no coefficients were coded
(:186-187); for inter pictures motion compensation ADD against the references
(MotionCompensator::CompensatePicture, :189-205, the second reference defaulting to the first);
then Picture::Clip (:207).  Output samples are value + 2^(depth-1) (set_frame_component,
libdirac_decoder/dirac_parser.cpp:159-226).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use this module.
"""
import numpy as np

from oracle import BlockParams, Oracle, chroma_shift


def decode_picture(cfg, pic, refs, ncb, oracle=None):
    """One picture.

    cfg: cformat, width, height, luma_depth, chroma_depth, wlt_depth, and for inter pictures
    mv_precision, xblen, yblen, xbsep, ybsep.  pic: intra, filter, zero_residual (optional),
    qindex (three int32 [ch][cw]), qidx and skip (three per-band arrays), cb_skip (three
    per-component flag arrays), me ({"mv": [mv1, mv2?], "mode", "dc", "split"}) for inter
    pictures.  refs: the reference pictures' decoded planes (one or two lists of three).
    ncb: per band (x, y) code blocks.  Returns the three decoded int16 planes."""
    orc = oracle or Oracle()
    xs, ys = chroma_shift(cfg["cformat"])
    w, h = cfg["width"], cfg["height"]
    sizes = [(w, h), (w >> xs, h >> ys), (w >> xs, h >> ys)]
    depth = cfg["wlt_depth"]
    intra = bool(pic["intra"])
    data = []
    for c in range(3):
        cw_, ch_ = sizes[c]
        if pic.get("zero_residual"):
            if intra:
                raise ValueError("intra pictures cannot have a zero residual")
            data.append(np.zeros((ch_, cw_), np.int16))
            continue
        coeff = orc.dequantise(intra, depth, pic["qindex"][c], pic["qidx"][c], pic["skip"][c], ncb, pic["cb_skip"][c])
        data.append(orc.dwt_backward(pic["filter"], depth, coeff, cw_, ch_))
    if not intra:
        me = pic["me"]
        xbsep, ybsep = cfg["xbsep"], cfg["ybsep"]
        bp = BlockParams(cfg["mv_precision"], cfg["xblen"], cfg["yblen"], xbsep, ybsep,
                         (w + 4 * xbsep - 1) // (4 * xbsep), (h + 4 * ybsep - 1) // (4 * ybsep))
        two = len(refs) > 1
        data = orc.motion_compensate(0, cfg["cformat"], data, refs[0], refs[1] if two else None, bp, me["mv"][0],
                                     me["mv"][1] if two else None, me["mode"], me["dc"], me["split"],
                                     cfg["luma_depth"], cfg["chroma_depth"])
    for c in range(3):
        orc.clip(data[c], cfg["luma_depth"] if c == 0 else cfg["chroma_depth"])
    return data


def output_samples(planes, luma_depth, chroma_depth):
    """set_frame_component: codec samples to unsigned output samples."""
    out = []
    for c, p in enumerate(planes):
        d = luma_depth if c == 0 else chroma_depth
        out.append((p.astype(np.int32) + (1 << (d - 1))).astype(np.uint8 if d <= 8 else np.uint16))
    return out


def decode_coded_sequence(cfg, enc, ncb, oracle=None):
    """Decodes, in coding order, the pictures an oracle_encoder.OracleEncoder coded (their
    quantised indices, band and code-block choices and motion data); returns {pnum: planes}."""
    orc = oracle or Oracle()
    out = {}
    for pn in enc.order:
        p = enc.pics[pn]
        r = p.result
        pic = {"intra": p.intra, "filter": r["filter"], "qindex": r["qindex"], "qidx": r["qidx"], "skip": r["skip"],
               "cb_skip": r["cb_skip"], "me": p.me}
        refs = [out[k] for k in p.refs] if not p.intra else None
        out[pn] = decode_picture(cfg, pic, refs, ncb, orc)
    return out
