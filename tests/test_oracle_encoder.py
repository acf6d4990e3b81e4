"""The oracle's restatement of the reference coding loop (oracle/oracle_encoder.py) against
the reference encoder itself: every locally decoded picture must be identical, for a plain
GOP, a GOP with a second I picture, the switch to P-only sub-groups, and cut detection at
B and P positions.  Fixtures: tests/golden/encode.npz (CRC-32 per plane, picture types),
made by tests/golden/make_golden.py through the reference's public encoder API."""
import os
import sys
import zlib

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import ENCODE_CASES, encode_inputs  # noqa: E402


def oracle_encode(case):
    from dirac_b200 import quant, synth
    from oracle_encoder import encode_sequence

    seq, cfg = encode_inputs(case)
    ocfg = {k: v for k, v in cfg.items() if k != "video_format"}
    ocfg.update(luma_depth=8, chroma_depth=8)
    frames = [[synth.to_signed(p) for p in f] for f in seq]
    return seq, cfg, encode_sequence(ocfg, frames, quant.band_weights, quant.code_blocks)


def recon_u8(pic):
    return [(p.astype(np.int32) + 128).astype(np.uint8) for p in pic.data]


@pytest.mark.parametrize("case", ENCODE_CASES, ids=[c[0] for c in ENCODE_CASES])
def test_oracle_encoder_matches_reference_fixtures(golden, case):
    g = golden("encode.npz")
    name = case[0]
    _, _, enc = oracle_encode(case)
    crc = np.array([[zlib.crc32(np.ascontiguousarray(p).tobytes()) for p in recon_u8(enc.pics[i])]
                    for i in range(len(enc.pics))], np.uint32)
    np.testing.assert_array_equal(crc, g[name + "_crc"])
    np.testing.assert_array_equal([int(enc.pics[i].intra) for i in range(len(enc.pics))], g[name + "_ptype"])


def test_oracle_encoder_matches_live_reference():
    from oracle import Reference, reference_encode

    if not Reference.available():
        pytest.skip("reference library not built here")
    seq, cfg, enc = oracle_encode(ENCODE_CASES[1])
    rec, ptype, _ = reference_encode(cfg, seq, freeze=True)
    for i in range(len(seq)):
        for c, p in enumerate(recon_u8(enc.pics[i])):
            np.testing.assert_array_equal(p, rec[i][c], err_msg=f"picture {i} component {c}")


def test_gop_structure_of_the_reconfigured_case():
    """Cut and P-only switch decisions of the restated loop, spelled out."""
    _, _, enc = oracle_encode(ENCODE_CASES[1])
    assert enc.order == [0, 1, 2, 3, 6, 4, 5, 9, 7, 8, 12, 10, 11, 13]
    assert enc.pics[3].cut and enc.pics[3].refs == [2]
    assert enc.pics[1].refs == [0] and enc.pics[2].refs == [1]
    assert enc.pics[6].refs == [3] and enc.pics[9].refs == [6, 3]


@pytest.mark.parametrize("case", [c for c in ENCODE_CASES if c[0] in ("reconfig", "cut_b")], ids=lambda c: c[0])
def test_code_picture_matches_the_coding_loop(case):
    """The oracle's single-picture coder (code_picture, which checks the picture batch) gives,
    for every picture of a sequence, what the coding loop gave it: the same reconstruction
    and residue results from the picture's original planes, its references' reconstructions
    and its motion data.  Covers intra, P, B and cut pictures."""
    from dirac_b200 import quant
    from oracle_encoder import code_picture

    _, cfg, enc = oracle_encode(case)
    c = enc.cfg
    for pn in enc.order:
        p = enc.pics[pn]
        pic = dict(cformat=c["cformat"], width=c["width"], height=c["height"], luma_depth=8, chroma_depth=8,
                   filter=c["intra_filter"] if p.intra else c["inter_filter"], wlt_depth=c["wlt_depth"],
                   intra=int(p.intra), is_b=int(p.is_b()), qf=c["qf"], cpd=c["cpd"], intra_ratio=p.ratio,
                   mv_precision=c["mv_precision"], xblen=c["xblen"], yblen=c["yblen"], xbsep=c["xbsep"],
                   ybsep=c["ybsep"])
        refs = None if p.intra else [enc.pics[r].data for r in p.refs]
        data, res = code_picture(pic, p.orig, quant.band_weights, quant.code_blocks, enc.orc, refs=refs,
                                 me=None if p.intra else p.me)
        for comp in range(3):
            np.testing.assert_array_equal(data[comp], p.data[comp], err_msg=f"picture {pn} component {comp}")
            for k in ("coeff", "qindex", "skip", "bits", "cb_skip"):
                np.testing.assert_array_equal(res[k][comp], p.result[k][comp], err_msg=f"picture {pn} {k}")
