"""Algorithmic bytes of the sequence encoder's stages: what each stage must move through HBM
at least once (the numerator of the roofline fractions bench.py reports).

Per picture of W x H luma samples, components (cw, ch) padded to the transform size:
  load             1 B (8-bit) or 2 B input read + 2 x 2 B (original and working planes) per sample
  dwt_forward      level 1: 2 B picture read + 4 B coefficient write per sample; deeper levels
                   8 B (read + write int32) per low-pass sample of that level
  dwt_inverse      the same in reverse
  quantisation     16 B per coefficient: the statistics read, the quantiser's read and in-place
                   write, and the quantised-index write
  mc_subtract      per sample: 2 B read + 2 B write of the picture plus 8 B per reference (the
  mc_add_clip      quarter-pel bilinear reads of the upconverted reference)
  upconvert        per reference picture: 2 B read + 8 B write per input sample
  motion_estimation  per inter picture: the pyramid of every picture involved built once
                   (2 B read + 0.5 B write per sample per level over the luma), the upconverted
                   original luma of each reference written (8 B per sample) and read by the
                   sub-pel search (8 B), and the luma of the picture and each reference read at
                   every pyramid level (2 B per sample per level, 4/3 overall)
"""


def dwt_bytes(cw, ch, depth):
    total = 0
    for lev in range(1, depth + 1):
        n = (cw >> (lev - 1)) * (ch >> (lev - 1))
        total += n * (6 if lev == 1 else 8)
    return total


def stage_bytes(params, infos):
    """Algorithmic bytes per stage for the pictures described by infos (encoder picture infos
    of one coded sequence)."""
    w, h = params["width"], params["height"]
    cf = params["cformat"]
    xs = 0 if cf == 0 else 1
    ys = 1 if cf == 2 else 0
    depth = params["wlt_depth"]
    mul = 1 << depth
    comps = [(w, h), (w >> xs, h >> ys), (w >> xs, h >> ys)]
    pad = [((a + mul - 1) // mul * mul, (b + mul - 1) // mul * mul) for a, b in comps]
    samples = sum(a * b for a, b in comps)
    coeffs = sum(a * b for a, b in pad)
    sb = 1 if params["luma_depth"] <= 8 and params["chroma_depth"] <= 8 else 2
    luma = w * h
    out = {k: 0 for k in ("load", "motion_estimation", "mc_subtract", "dwt_forward", "quantisation",
                          "dwt_inverse", "mc_add_clip", "upconvert")}
    refs_used = set()
    for i in infos:
        out["load"] += samples * (sb + 4)
        d = sum(dwt_bytes(a, b, depth) for a, b in pad)
        out["dwt_forward"] += d
        out["dwt_inverse"] += d
        out["quantisation"] += 16 * coeffs
        nref = i["num_refs"]
        if nref and not i["intra"]:
            mc = samples * (4 + 8 * nref)
            out["mc_subtract"] += mc
            out["mc_add_clip"] += mc
        else:
            out["mc_add_clip"] += samples * 4  # the clip alone
        if nref:
            out["motion_estimation"] += int(luma * (2.5 * 4 / 3) * (1 + nref) + luma * 16 * nref
                                            + luma * 2 * (4 / 3) * (1 + nref))
            for r in (i["ref1"], i["ref2"]):
                if r >= 0:
                    refs_used.add(r)
    out["upconvert"] = len(refs_used) * samples * 10
    return out


def decode_bytes(params, infos, int16_pictures=0):
    """Algorithmic bytes per stage of the device decoder for the pictures described by infos
    (coded pictures in coding order): dequantisation 8 B per coefficient (int32 index read,
    coefficient write; 6 B in the int16_pictures whose indices are int16), the inverse
    transform, motion compensation ADD with the clip (or the clip alone for intra pictures) and
    the upconversion of every reference picture, as above."""
    enc = stage_bytes(params, infos)
    w, h = params["width"], params["height"]
    cf = params["cformat"]
    xs = 0 if cf == 0 else 1
    ys = 1 if cf == 2 else 0
    mul = 1 << params["wlt_depth"]
    comps = [(w, h), (w >> xs, h >> ys), (w >> xs, h >> ys)]
    coeffs = sum((a + mul - 1) // mul * mul * ((b + mul - 1) // mul * mul) for a, b in comps)
    samples = sum(a * b for a, b in comps)
    refs = {r for i in infos if not i["intra"] for r in (i["ref1"], i["ref2"]) if r >= 0}
    return {"dequantisation": coeffs * (8 * len(infos) - 2 * int16_pictures), "dwt_inverse": enc["dwt_inverse"],
            "mc_add_clip": enc["mc_add_clip"], "upconvert": len(refs) * samples * 10}
