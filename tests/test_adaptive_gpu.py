"""The device encoder as a drop-in for the stock reference encoder: each picture coded with the
encoder's whole entropy-correction state (dgpu_encoder_code_next_adaptive), its quantised
subbands then arithmetic-coded on the host (dgpu_code_bands_host) and the state adapted from
the byte counts (dgpu_entropy_update), as the reference's CompCompressor does.  The locally
decoded pictures equal the stock reference encoder's, adaptive factors included
(tests/golden/adaptive.npz, made through the reference's public encoder API)."""
import os
import sys
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import ENCODE_CASES, encode_inputs  # noqa: E402


def adaptive_encode(seq, cfg, vlc=False):
    """Codes seq with the device encoder and the host band coder adapting the entropy-correction
    state picture by picture (the stock reference encoder's loop; with vlc the variable-length
    coder, whose whole bytes the reference's update takes); returns the locally decoded output
    planes and intra flags by picture number."""
    from dirac_b200 import encoder as E
    from dirac_b200 import quant
    from dirac_b200.encoder import SequenceEncoder
    from dirac_b200.entropy import EntropyCorrector, code_bands

    depth = cfg["wlt_depth"]
    ncb = quant.code_blocks(depth, cfg["width"], cfg["height"])
    ec = EntropyCorrector(depth)
    enc = SequenceEncoder(cfg, max_pictures=len(seq))
    for f in seq:
        enc.load(f)
    enc.end_sequence()
    outputs, ptype = {}, {}
    while True:
        info = enc.code_next(ecf_state=ec.state)
        if info is None:
            break
        pn = info["pnum"]
        xs = 1
        for c in range(3):
            bands = enc.read(pn, E.BANDS, c).reshape(-1, 3)
            q = enc.read(pn, E.QINDEX, c)
            cw = ((cfg["width"] >> (xs if c else 0)) + (1 << depth) - 1) >> depth << depth
            coded = code_bands(info["intra"], depth, [q.reshape(-1, cw)], [bands], [ncb],
                               [enc.read(pn, E.CBSKIP, c)], vlc=vlc)
            counts = coded[2][0] // 8 if vlc else coded[1][0]
            ec.update(info["intra"], info["is_b"], c, bands[:, 1], bands[:, 2], counts)
        outputs[pn] = [enc.read(pn, E.OUTPUT, c) for c in range(3)]
        ptype[pn] = info["intra"]
    enc.close()
    return outputs, ptype


@pytest.mark.parametrize("case", ENCODE_CASES, ids=[c[0] for c in ENCODE_CASES])
def test_device_encoder_with_host_coder_matches_stock_reference(gpu, golden, case):
    from test_encoder_gpu import encoder_params

    seq, rcfg = encode_inputs(case)
    outputs, ptype = adaptive_encode(seq, encoder_params(rcfg))
    g = golden("adaptive.npz")
    crc = np.array([[zlib.crc32(np.ascontiguousarray(outputs[i][c]).tobytes()) for c in range(3)]
                    for i in range(len(seq))], np.uint32)
    np.testing.assert_array_equal(crc, g[case[0] + "_crc"])
    np.testing.assert_array_equal([ptype[i] for i in range(len(seq))], g[case[0] + "_ptype"])


def read_coded(enc, info, cfg):
    """A coded picture's quantised indices, band tables and code-block flags (host copies)."""
    from dirac_b200 import encoder as E

    depth = cfg["wlt_depth"]
    pn = info["pnum"]
    out = []
    for c in range(3):
        cw = ((cfg["width"] >> (1 if c else 0)) + (1 << depth) - 1) >> depth << depth
        out.append((enc.read(pn, E.QINDEX, c).reshape(-1, cw), enc.read(pn, E.BANDS, c).reshape(-1, 3),
                    enc.read(pn, E.CBSKIP, c)))
    return out


@pytest.mark.parametrize("case", [ENCODE_CASES[0], ENCODE_CASES[3]], ids=[ENCODE_CASES[0][0], ENCODE_CASES[3][0]])
def test_pipelined_host_coding_matches_stock_reference(gpu, golden, case):
    """Picture n's subbands arithmetic-coded on a host thread while the device prepares picture
    n + 1 (estimation, compensation, transform); n + 1's quantisers chosen after n's byte counts
    have updated the factors.  Same pictures as the stock reference encoder."""
    from concurrent.futures import ThreadPoolExecutor

    from dirac_b200 import encoder as E
    from dirac_b200 import quant
    from dirac_b200.encoder import SequenceEncoder
    from dirac_b200.entropy import EntropyCorrector, code_bands
    from test_encoder_gpu import encoder_params

    seq, rcfg = encode_inputs(case)
    cfg = encoder_params(rcfg)
    depth = cfg["wlt_depth"]
    ncb = quant.code_blocks(depth, cfg["width"], cfg["height"])
    ec = EntropyCorrector(depth)
    enc = SequenceEncoder(cfg, max_pictures=len(seq))
    for f in seq:
        enc.load(f)
    enc.end_sequence()

    def code_and_adapt(info, comps):
        for c, (q, bands, cbs) in enumerate(comps):
            _, per = code_bands(info["intra"], depth, [q], [bands], [ncb], [cbs])
            ec.update(info["intra"], info["is_b"], c, bands[:, 1], bands[:, 2], per[0])

    outputs, pending = {}, None
    with ThreadPoolExecutor(1) as ex:
        while True:
            fut = ex.submit(code_and_adapt, *pending) if pending else None
            nxt = enc.prepare_next()
            if fut:
                fut.result()
            if nxt is None:
                break
            info = enc.finish_next(ecf_state=ec.state)
            assert info["pnum"] == nxt["pnum"] and info["intra"] == nxt["intra"]
            outputs[info["pnum"]] = [enc.read(info["pnum"], E.OUTPUT, c) for c in range(3)]
            pending = (info, read_coded(enc, info, cfg))
    enc.close()
    g = golden("adaptive.npz")
    crc = np.array([[zlib.crc32(np.ascontiguousarray(outputs[i][c]).tobytes()) for c in range(3)]
                    for i in range(len(seq))], np.uint32)
    np.testing.assert_array_equal(crc, g[case[0] + "_crc"])


@pytest.mark.parametrize("case", ENCODE_CASES, ids=[c[0] for c in ENCODE_CASES])
def test_device_encoder_with_vlc_host_coder_matches_stock_reference(gpu, golden, case):
    """The stock -use_vlc reference encoder: coefficients coded by the variable-length host coder
    (dgpu_code_bands_vlc_host), the factors adapted from its whole-byte counts."""
    from test_encoder_gpu import encoder_params

    seq, rcfg = encode_inputs(case)
    outputs, ptype = adaptive_encode(seq, encoder_params(rcfg), vlc=True)
    g = golden("adaptive.npz")
    crc = np.array([[zlib.crc32(np.ascontiguousarray(outputs[i][c]).tobytes()) for c in range(3)]
                    for i in range(len(seq))], np.uint32)
    np.testing.assert_array_equal(crc, g[case[0] + "_vlc_crc"])
    np.testing.assert_array_equal([ptype[i] for i in range(len(seq))], g[case[0] + "_vlc_ptype"])


def test_hd1080_with_host_coder_matches_stock_reference(gpu, golden):
    """The bench's 1080p workload (first 10 frames of its sequence) coded as the stock reference
    encoder codes it: device encoder, host band coder, factors adapted after every picture.
    Every locally decoded plane equals the stock reference encoder's (hd1080.npz, adaptive),
    which its own decoder reproduces from its bitstream."""
    from make_golden import hd_inputs
    from test_encoder_gpu import encoder_params

    seq, rcfg = hd_inputs()
    outputs, ptype = adaptive_encode(seq, encoder_params(rcfg))
    g = golden("hd1080.npz")
    crc = np.array([[zlib.crc32(np.ascontiguousarray(outputs[i][c]).tobytes()) for c in range(3)]
                    for i in range(len(seq))], np.uint32)
    np.testing.assert_array_equal([ptype[i] for i in range(len(seq))], g["adaptive_ptype"])
    np.testing.assert_array_equal(crc, g["adaptive_crc"])
    np.testing.assert_array_equal(g["adaptive_crc"], g["adaptive_decode_crc"])


def _pipelined_outputs(seq, cfg, native=False):
    from dirac_b200 import encoder as E
    from dirac_b200.adaptive import AdaptiveCoder
    from dirac_b200.encoder import SequenceEncoder

    enc = SequenceEncoder(cfg, max_pictures=len(seq))
    for f in seq:
        enc.load(f)
    enc.end_sequence()
    coder = AdaptiveCoder(enc, cfg)
    outputs = {}
    coded = {}

    def fin(info):
        outputs[info["pnum"]] = [enc.read(info["pnum"], E.OUTPUT, c) for c in range(3)]

    def done(info, got, data, per):
        coded[info["pnum"]] = (zlib.crc32(data.tobytes()), [int(x) for p in per for x in p])

    if native:
        # every picture keeps its slot (max_pictures = the sequence), so outputs are read after
        infos, data, bb = coder.run_native(max_pictures=len(seq))
        coded["d2h_bytes"] = coder.d2h_bytes
        for info, d, b in zip(infos, data, bb):
            fin(info)
            coded[info["pnum"]] = (zlib.crc32(d.tobytes()), [int(x) for x in b.ravel()])
    else:
        infos = coder.run(on_finished=fin, on_coded=done)
    coder.close()
    enc.close()
    crc = np.array([[zlib.crc32(np.ascontiguousarray(outputs[i][c]).tobytes()) for c in range(3)]
                    for i in range(len(seq))], np.uint32)
    return crc, infos, coded


@pytest.mark.parametrize("case", [ENCODE_CASES[0], "hd1080"], ids=[ENCODE_CASES[0][0], "hd1080"])
def test_kind_pipelined_coder_matches_stock_reference(gpu, golden, case):
    """AdaptiveCoder: a picture waits only for the host coding of the last picture of its own
    kind (the factors it reads), so host coding overlaps the device work of the pictures after
    it.  Every locally decoded plane equals the stock reference encoder's, and the coded band
    bytes equal the serial loop's (one picture coded and adapted before the next)."""
    from test_encoder_gpu import encoder_params

    if case == "hd1080":
        from make_golden import hd_inputs

        seq, rcfg = hd_inputs()
        want = golden("hd1080.npz")["adaptive_crc"]
    else:
        seq, rcfg = encode_inputs(case)
        want = golden("adaptive.npz")[case[0] + "_crc"]
    cfg = encoder_params(rcfg)
    crc, infos, coded = _pipelined_outputs(seq, cfg)
    np.testing.assert_array_equal(crc, want)
    assert sorted(coded) == sorted(i["pnum"] for i in infos) and len(coded) == len(seq)
    # the library's own pipeline (dgpu_encoder_code_adaptive): same pictures, same coded bytes
    ncrc, ninfos, ncoded = _pipelined_outputs(seq, cfg, native=True)
    np.testing.assert_array_equal(ncrc, want)
    assert [i["pnum"] for i in ninfos] == [i["pnum"] for i in infos]
    d2h = ncoded.pop("d2h_bytes")
    assert ncoded == coded
    # inter pictures' indices went as int16: fewer bytes than every picture's int32 indices
    n_idx = sum(a * b for a, b in _padded(cfg))
    n_inter = sum(1 for i in ninfos if not i["intra"])
    assert n_inter > 0 and d2h <= 4 * n_idx * len(ninfos) - 2 * n_idx * n_inter + 64 * len(ninfos) + \
        _motion_bytes(cfg) * len(ninfos)


def _padded(cfg):
    m = 1 << cfg["wlt_depth"]
    out = []
    for c in range(3):
        w = cfg["width"] >> (0 if c == 0 or cfg["cformat"] == 0 else 1)
        h = cfg["height"] >> (1 if c and cfg["cformat"] == 2 else 0)
        out.append(((h + m - 1) // m * m, (w + m - 1) // m * m))
    return out


def _motion_bytes(cfg):
    """Upper bound of one picture's motion-data bytes (two vector sets, modes, DCs, splits)."""
    xsb = (cfg["width"] + 4 * cfg["xbsep"] - 1) // (4 * cfg["xbsep"])
    ysb = (cfg["height"] + 4 * cfg["ybsep"] - 1) // (4 * cfg["ybsep"])
    nb = 16 * xsb * ysb
    return nb * (2 * 4 + 1 + 3 * 2) + xsb * ysb


def test_native_pipeline_wide_residues_match_python_pipeline(gpu):
    """14-bit noise: inter residues whose coefficients exceed 16 bits, so some inter pictures'
    indices go as int32 and others may go as int16.  The library's pipeline codes the same bytes
    and pictures as the Python pipeline, which reads every picture's int32 indices."""
    from test_encoder_gpu import encoder_params

    rng = np.random.default_rng(23)
    w, h, n = 128, 96, 7
    seq = [tuple(rng.integers(0, 1 << 14, size=(h >> (c > 0), w >> (c > 0))).astype(np.uint16) for c in range(3))
           for _ in range(n)]
    cfg = encoder_params(dict(cformat=2, width=w, height=h, qf=9.0, l1_sep=3, num_l1=1, cpd=20.0, xblen=12,
                              yblen=12, xbsep=8, ybsep=8, mv_precision=2, intra_filter=1, inter_filter=4,
                              wlt_depth=4))
    cfg.update(luma_depth=14, chroma_depth=14)
    crc, infos, coded = _pipelined_outputs(seq, cfg)
    ncrc, ninfos, ncoded = _pipelined_outputs(seq, cfg, native=True)
    ncoded.pop("d2h_bytes")
    np.testing.assert_array_equal(ncrc, crc)
    assert [i["pnum"] for i in ninfos] == [i["pnum"] for i in infos]
    assert ncoded == coded
