"""The device sequence encoder (dgpu_encoder_*) against the oracle's restatement of the
reference coding loop, picture by picture and bit for bit: picture types and references,
motion vectors, modes, DC values, splits, quantiser choices, skip flags, bit estimates,
code-block skips, quantised indices, reconstructed coefficients and reconstructed pictures;
and the locally decoded pictures against the reference encoder's own (golden CRC-32s)."""
import os
import sys
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import ENCODE_CASES, encode_inputs  # noqa: E402


def encoder_params(cfg):
    p = {k: v for k, v in cfg.items() if k != "video_format"}
    p.update(luma_depth=8, chroma_depth=8)
    return p


def run_device(gpu, seq, cfg, max_pictures=None, ecf_fn=None, read_each=False):
    from dirac_b200.encoder import SequenceEncoder
    from dirac_b200 import encoder as E

    enc = SequenceEncoder(encoder_params(cfg), max_pictures=max_pictures or len(seq))
    infos, results = [], {}

    def drain():
        while True:
            info = enc.code_next(ecf_fn(enc) if ecf_fn is not None else None)
            if info is None:
                return
            infos.append(info)
            if read_each:
                results[info["pnum"]] = read_all(enc, info["pnum"])

    # the reference encoder's application loop: load a picture, code what can be coded
    for f in seq:
        enc.load(f)
        if max_pictures is not None:
            drain()
    enc.end_sequence()
    drain()
    if not read_each:
        for i in infos:
            results[i["pnum"]] = read_all(enc, i["pnum"])
    enc.close()
    return infos, results


def read_all(enc, pnum):
    from dirac_b200 import encoder as E

    r = {}
    for name, what in (("recon", E.RECON), ("coeff", E.COEFF), ("qindex", E.QINDEX), ("bands", E.BANDS),
                       ("cb_skip", E.CBSKIP), ("output", E.OUTPUT)):
        r[name] = [enc.read(pnum, what, c) for c in range(3)]
    for name, what in (("mv", E.MV), ("mode", E.MODE), ("dc", E.DC), ("split", E.SPLIT)):
        r[name] = enc.read(pnum, what)
    return r


def oracle_run(cfg, seq, ecf_fn=None):
    from dirac_b200 import quant, synth
    from oracle_encoder import encode_sequence

    frames = [[synth.to_signed(p) for p in f] for f in seq]
    return encode_sequence(encoder_params(cfg), frames, quant.band_weights, quant.code_blocks, ecf_fn=ecf_fn)


def compare(infos, results, oenc):
    assert [i["pnum"] for i in infos] == oenc.order
    for info in infos:
        pn = info["pnum"]
        p = oenc.pics[pn]
        r = results[pn]
        msg = f"picture {pn}"
        assert bool(info["intra"]) == p.intra and bool(info["cut"]) == p.cut, msg
        refs = [x for x in (info["ref1"], info["ref2"]) if x >= 0]
        assert refs == p.refs, msg
        if p.me is not None and (not p.intra or p.cut):
            assert info["intra_ratio"] == p.ratio, msg
            nref = len(p.refs)
            np.testing.assert_array_equal(r["mv"].reshape(p.me["mv"].shape[:1] + (-1, 2))[:nref],
                                          p.me["mv"].reshape(nref, -1, 2), err_msg=msg)
            np.testing.assert_array_equal(r["mode"], p.me["mode"].ravel(), err_msg=msg)
            np.testing.assert_array_equal(r["dc"], p.me["dc"].ravel(), err_msg=msg)
            np.testing.assert_array_equal(r["split"], p.me["split"].ravel(), err_msg=msg)
        res = p.result
        for c in range(3):
            cm = f"{msg} component {c}"
            np.testing.assert_array_equal(r["coeff"][c], res["coeff"][c].ravel(), err_msg=cm)
            np.testing.assert_array_equal(r["qindex"][c], res["qindex"][c].ravel(), err_msg=cm)
            b = r["bands"][c].reshape(-1, 3)
            sk = res["skip"][c]
            np.testing.assert_array_equal(b[:, 1], sk, err_msg=cm)
            np.testing.assert_array_equal(b[:, 0][sk == 0], res["qidx"][c][sk == 0], err_msg=cm)
            np.testing.assert_array_equal(b[:, 2], res["bits"][c], err_msg=cm)
            np.testing.assert_array_equal(r["cb_skip"][c], res["cb_skip"][c], err_msg=cm)
            np.testing.assert_array_equal(r["recon"][c], p.data[c].ravel(), err_msg=cm)
            assert np.float32(info["lambda"][c]) == np.float32(res["lambda"][c]), cm


@pytest.mark.parametrize("case", ENCODE_CASES, ids=[c[0] for c in ENCODE_CASES])
def test_encoder_matches_oracle_and_reference(gpu, golden, case):
    seq, cfg = encode_inputs(case)
    infos, results = run_device(gpu, seq, cfg)
    compare(infos, results, oracle_run(cfg, seq))
    g = golden("encode.npz")
    crc = np.array([[zlib.crc32(np.ascontiguousarray(results[i]["output"][c]).tobytes()) for c in range(3)]
                    for i in range(len(seq))], np.uint32)
    np.testing.assert_array_equal(crc, g[case[0] + "_crc"])


def test_encoder_slot_reuse(gpu):
    """A 30-picture sequence through 20 picture slots gives the same pictures as the oracle
    (results read right after each picture is coded)."""
    from dirac_b200 import synth

    seq = synth.make_sequence(176, 144, 30, n_rects=5, vmax=5, seed=31)
    cfg = dict(cformat=2, width=176, height=144, qf=6.0, l1_sep=3, num_l1=4, cpd=20.0, xblen=12, yblen=12, xbsep=8,
               ybsep=8, mv_precision=2, intra_filter=1, inter_filter=0, wlt_depth=3)
    infos, results = run_device(gpu, seq, cfg, max_pictures=20, read_each=True)
    compare(infos, results, oracle_run(cfg, seq))


@pytest.mark.parametrize("mode", [1, 2], ids=["sleep", "yield"])
def test_encoder_host_wait_modes(gpu, mode):
    """dgpu_set_blocking_waits changes only how host threads wait for the device: a sequence
    coded with waits that sleep on a blocking-sync event, or poll and yield, gives the oracle's
    pictures."""
    from dirac_b200 import synth

    lib = gpu.load()
    seq = synth.make_sequence(176, 144, 8, n_rects=5, vmax=5, seed=37)
    cfg = dict(cformat=2, width=176, height=144, qf=6.0, l1_sep=3, num_l1=2, cpd=20.0, xblen=12, yblen=12, xbsep=8,
               ybsep=8, mv_precision=2, intra_filter=1, inter_filter=0, wlt_depth=3)
    try:
        assert lib.dgpu_set_blocking_waits(mode) == 0
        infos, results = run_device(gpu, seq, cfg, read_each=True)
    finally:
        assert lib.dgpu_set_blocking_waits(0) == 0
    compare(infos, results, oracle_run(cfg, seq))


def test_encoder_caller_entropy_factors(gpu):
    """Entropy-correction factors supplied per picture by the caller (as the host arithmetic
    coder's adaptation would) reach the quantiser choice exactly as in the oracle."""
    from dirac_b200 import synth

    seq = synth.make_sequence(176, 144, 8, n_rects=5, vmax=5, seed=32)
    cfg = dict(cformat=2, width=176, height=144, qf=8.0, l1_sep=3, num_l1=19, cpd=20.0, xblen=12, yblen=12, xbsep=8,
               ybsep=8, mv_precision=2, intra_filter=6, inter_filter=0, wlt_depth=4)
    nb = 13

    def factors(pnum):
        rng = np.random.default_rng(1000 + pnum)
        return rng.uniform(0.5, 1.5, size=(3, nb)).astype(np.float32)

    def dev_ecf(enc):
        # all pictures are loaded before coding starts, so every call codes the oracle's next
        # picture in coding order
        if dev_ecf.k >= len(oenc.order):
            return None  # the final call, which codes nothing
        pn = oenc.order[dev_ecf.k]
        dev_ecf.k += 1
        return factors(pn)

    dev_ecf.k = 0

    oenc = oracle_run(cfg, seq, ecf_fn=lambda p: factors(p.pnum))
    infos, results = run_device(gpu, seq, cfg, ecf_fn=dev_ecf)
    compare(infos, results, oenc)


@pytest.mark.parametrize("cformat,depth", [(1, 10), (0, 8), (2, 12)])
def test_encoder_formats_and_depths(gpu, cformat, depth):
    """4:2:2 10-bit, 4:4:4 8-bit and 4:2:0 12-bit sequences (16-bit input samples above 8
    bits) through the device encoder equal the oracle's restatement, picture by picture."""
    from dirac_b200 import quant, synth
    from oracle_encoder import encode_sequence

    w, h, n = 176, 144, 7
    chroma = {0: "444", 1: "422", 2: "420"}[cformat]
    seq = synth.make_sequence(w, h, n, n_rects=5, vmax=5, seed=40 + cformat, bit_depth=depth, chroma=chroma)
    cfg = dict(cformat=cformat, width=w, height=h, luma_depth=depth, chroma_depth=depth, qf=6.5, l1_sep=3,
               num_l1=19, cpd=20.0, xblen=12, yblen=12, xbsep=8, ybsep=8, mv_precision=2, intra_filter=6,
               inter_filter=2, wlt_depth=3)
    from dirac_b200.encoder import SequenceEncoder

    enc = SequenceEncoder(cfg, max_pictures=n)
    infos = enc.encode(seq)
    results = {i["pnum"]: read_all(enc, i["pnum"]) for i in infos}
    enc.close()
    frames = [[synth.to_signed(p, depth) for p in f] for f in seq]
    oenc = encode_sequence(cfg, frames, quant.band_weights, quant.code_blocks)
    compare(infos, results, oenc)
    off = 1 << (depth - 1)
    for i in range(n):
        for c in range(3):
            np.testing.assert_array_equal(results[i]["output"][c],
                                          (oenc.pics[i].data[c].astype(np.int32) + off).ravel())


def test_encoder_group_estimation(gpu, golden):
    """Three sequences (a switch to P-only sub-groups, a cut at a B position, a cut at a P
    position) coded by three encoders whose motion estimation runs as one group batch: every
    picture equals the oracle's, and the locally decoded pictures the reference encoder's."""
    from dirac_b200.encoder import EncoderGroup, SequenceEncoder

    cases = [c for c in ENCODE_CASES if c[0] in ("reconfig", "cut_b", "cut_p")]
    inputs = [encode_inputs(c) for c in cases]
    encs = [SequenceEncoder(encoder_params(cfg), max_pictures=len(seq)) for seq, cfg in inputs]
    group = EncoderGroup(encs)
    for enc, (seq, _) in zip(encs, inputs):
        for f in seq:
            enc.load(f)
        enc.end_sequence()
    n = group.estimate()
    assert n == sum(len(seq) - 1 for seq, _ in inputs)  # every picture but the first is inter at first
    assert group.estimate() == 0  # nothing left to estimate
    g = golden("encode.npz")
    for case, enc, (seq, cfg) in zip(cases, encs, inputs):
        infos = []
        while True:
            info = enc.code_next()
            if info is None:
                break
            infos.append(info)
        results = {i["pnum"]: read_all(enc, i["pnum"]) for i in infos}
        compare(infos, results, oracle_run(cfg, seq))
        crc = np.array([[zlib.crc32(np.ascontiguousarray(results[i]["output"][c]).tobytes()) for c in range(3)]
                        for i in range(len(seq))], np.uint32)
        np.testing.assert_array_equal(crc, g[case[0] + "_crc"])
    group.close()
    for enc in encs:
        enc.close()


def test_encoder_group_rejects_mixed_geometry(gpu):
    from dirac_b200 import _lib
    from dirac_b200.encoder import EncoderGroup, SequenceEncoder

    _, cfg = encode_inputs(ENCODE_CASES[1])
    a = SequenceEncoder(encoder_params(cfg), max_pictures=4)
    other = dict(encoder_params(cfg), width=352, height=288)
    b = SequenceEncoder(other, max_pictures=4)
    with pytest.raises(_lib.DgpuError):
        EncoderGroup([a, b])
    with pytest.raises(_lib.DgpuError):
        EncoderGroup([a, a])
    a.close()
    b.close()


def test_encoder_hd1080_matches_reference(gpu, golden):
    """The bench's 1080p coding workload (HD1080P50 GOP, QF 7, DAUB9_7 / DD9_7 depth 4, OBMC
    16/12, quarter-pel): the first 10 frames of its sequence coded by the device encoder with the
    initial entropy-correction factors, every locally decoded plane equal to the reference
    encoder's (tests/golden/hd1080.npz, frozen factors), picture types included."""
    from make_golden import hd_inputs

    seq, cfg = hd_inputs()
    infos, results = run_device(gpu, seq, cfg)
    g = golden("hd1080.npz")
    crc = np.array([[zlib.crc32(np.ascontiguousarray(results[i]["output"][c]).tobytes()) for c in range(3)]
                    for i in range(len(seq))], np.uint32)
    np.testing.assert_array_equal([int(i["intra"]) for i in sorted(infos, key=lambda i: i["pnum"])],
                                  g["frozen_ptype"])
    np.testing.assert_array_equal(crc, g["frozen_crc"])
