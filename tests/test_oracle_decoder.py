"""The oracle's restatement of the reference decoder's picture decoding (oracle/oracle_decoder.py,
orc_dequantise) against the reference: decoding what the restated encoder coded (quantised
indices, band quantisers and skips, code-block skips, motion data) must give the encoder's
locally decoded pictures and output samples equal to the reference decoder's own decode of the
reference encoder's bitstream (tests/golden/decode.npz, made through the reference's public
encoder and decoder APIs; equal to the reference encoder's local decode, encode.npz)."""
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
    return ocfg, encode_sequence(ocfg, frames, quant.band_weights, quant.code_blocks)


@pytest.mark.parametrize("case", ENCODE_CASES, ids=[c[0] for c in ENCODE_CASES])
def test_oracle_decoder_round_trip(golden, oracle, case):
    from dirac_b200 import quant
    from oracle_decoder import decode_coded_sequence, output_samples

    cfg, enc = oracle_encode(case)
    ncb = quant.code_blocks(cfg["wlt_depth"], cfg["width"], cfg["height"])
    dec = decode_coded_sequence(cfg, enc, ncb, oracle)
    crc = []
    for pn in range(len(enc.pics)):
        for c in range(3):
            np.testing.assert_array_equal(dec[pn][c], enc.pics[pn].data[c], err_msg=f"picture {pn} component {c}")
        crc.append([zlib.crc32(np.ascontiguousarray(p).tobytes()) for p in output_samples(dec[pn], 8, 8)])
    np.testing.assert_array_equal(np.array(crc, np.uint32), golden("decode.npz")[case[0] + "_crc"])
    np.testing.assert_array_equal(golden("decode.npz")[case[0] + "_crc"], golden("encode.npz")[case[0] + "_crc"])


def test_oracle_decoder_matches_live_reference_decoder(oracle):
    """The oracle's decode against the reference decoder's, sample for sample, on the
    reference encoder's own bitstream of the reconfigured sequence."""
    from dirac_b200 import quant
    from oracle import Reference, reference_decode, reference_encode_stream
    from oracle_decoder import decode_coded_sequence, output_samples

    if not Reference.available():
        pytest.skip("reference library not built here")
    seq, rcfg = encode_inputs(ENCODE_CASES[1])
    _, _, stream = reference_encode_stream(rcfg, seq, freeze=True)
    ref = reference_decode(stream, rcfg["width"], rcfg["height"], rcfg["cformat"], len(seq))
    cfg, enc = oracle_encode(ENCODE_CASES[1])
    dec = decode_coded_sequence(cfg, enc, quant.code_blocks(cfg["wlt_depth"], cfg["width"], cfg["height"]), oracle)
    for pn in range(len(seq)):
        for c, p in enumerate(output_samples(dec[pn], 8, 8)):
            np.testing.assert_array_equal(p, ref[pn][c], err_msg=f"picture {pn} component {c}")


def test_dequantise_values(oracle):
    """DecodeVal's arithmetic on a hand-checked band: qf4(8) = 16, intra offset 8, inter 6."""
    depth = 1
    q = np.zeros((4, 4), np.int32)
    q[0, 2] = 3     # band 3 (HL, top-right), inter: (3 * 16 + 6 + 2) >> 2 = 14
    q[1, 3] = -1    # (16 + 6 + 2) >> 2 = 6, negated
    q[2, 0] = 5     # band 2 (LH) skipped: 0
    ncb = [1, 1] * 4
    out = oracle.dequantise(0, depth, q, [8, 8, 8, 8], [0, 1, 0, 0], ncb, np.zeros(4, np.uint8))
    assert out[0, 2] == 14 and out[1, 3] == -6 and out[2, 0] == 0
    assert np.count_nonzero(out) == 2


def test_dequantise_intra_dc_prediction(oracle):
    """Intra DC band (depth 1: the 2 x 2 top-left band): residues plus the floor-division
    mean of the left, top-left and top reconstructed values (GetPrediction)."""
    q = np.zeros((4, 4), np.int32)
    q[0, 0], q[0, 1], q[1, 0], q[1, 1] = 2, -1, 1, 0      # qidx 0: qf4 4, intra offset 1
    ncb = [1, 1] * 4
    out = oracle.dequantise(1, 1, q, [0, 0, 0, 0], [0, 0, 0, 0], ncb, np.zeros(4, np.uint8))
    # values (q * 4 + 3) >> 2 = q for |q| >= 1; a = 2; b = -1 + a = 1; c = 1 + a = 3;
    # d = 0 + floor((c + a + b + 1) / 3) = floor(7 / 3) = 2
    assert out[0, 0] == 2 and out[0, 1] == 1 and out[1, 0] == 3 and out[1, 1] == 2


def test_dequantise_rejects_bad_quantiser(oracle):
    q = np.zeros((4, 4), np.int32)
    with pytest.raises(ValueError):
        oracle.dequantise(0, 1, q, [120, 0, 0, 0], [0, 0, 0, 0], [1, 1] * 4, np.zeros(4, np.uint8))
