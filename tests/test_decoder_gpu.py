"""The device decoder (dgpu_decoder_*) and the dequantisation stage (dgpu_dequantise_batch)
against the oracle and the reference.

Round trip: what the device encoder coded (quantised indices, band quantisers and skips,
code-block skips, motion data) decoded by the device decoder in coding order gives, bit for
bit, the encoder's locally decoded pictures and reconstructed coefficients, and output
samples equal to the reference decoder's decode of the reference encoder's bitstream (golden
CRC-32s); the same pictures decoded by the
oracle's restatement of the reference decoder agree.  The stage alone is checked against
orc_dequantise on random indices, skips and quantisers, intra and inter, depths 1-5."""
import os
import sys
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import ENCODE_CASES, encode_inputs  # noqa: E402


def encoded(gpu, case=None, cfg=None, seq=None):
    """Codes a sequence with the device encoder; returns (parameters, infos in coding order,
    every picture's results)."""
    from dirac_b200.encoder import SequenceEncoder
    from test_encoder_gpu import encoder_params, read_all

    if case is not None:
        seq, cfg = encode_inputs(case)
        cfg = encoder_params(cfg)
    enc = SequenceEncoder(cfg, max_pictures=len(seq))
    infos = enc.encode(seq)
    results = {i["pnum"]: read_all(enc, i["pnum"]) for i in infos}
    enc.close()
    return cfg, infos, results


def motion_of(results, info, device=False):
    import torch

    r = results[info["pnum"]]
    nref = info["num_refs"]
    mv = r["mv"].reshape(nref, -1, 2)
    m = {"mv": [mv[k] for k in range(nref)], "mode": r["mode"], "dc": r["dc"], "split": r["split"]}
    if device:
        m = {"mv": [torch.from_numpy(np.ascontiguousarray(v)).cuda() for v in m["mv"]],
             **{k: torch.from_numpy(np.ascontiguousarray(m[k])).cuda() for k in ("mode", "dc", "split")}}
    return m


def padded_shapes(cfg):
    """(ch, cw) of the three components' coefficient arrays."""
    m = 1 << cfg["wlt_depth"]
    out = []
    for c in range(3):
        w = cfg["width"] >> (0 if c == 0 or cfg["cformat"] == 0 else 1)
        h = cfg["height"] >> (1 if c and cfg["cformat"] == 2 else 0)
        out.append(((h + m - 1) // m * m, (w + m - 1) // m * m))
    return out


def decode_all(cfg, infos, results, device=False, max_pictures=None, release=False, idx16=False):
    """Decodes the coded pictures in coding order; with release, drops each picture once no
    later picture references it (after reading its results); with idx16, the indices go as
    int16 arrays (index_bits 16)."""
    import torch

    from dirac_b200.decoder import SequenceDecoder, decoder_params

    P = decoder_params(cfg)
    dec = SequenceDecoder(P, max_pictures=max_pictures or len(infos))
    shapes = padded_shapes(cfg)
    out = {}
    for k, info in enumerate(infos):
        pn = info["pnum"]
        r = results[pn]
        q = [r["qindex"][c].reshape(shapes[c]) for c in range(3)]
        if idx16:
            assert all(np.abs(a).max() <= 32767 for a in q)
            q = [a.astype(np.int16) for a in q]
        cbs = r["cb_skip"]
        if device:
            q = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in q]
            cbs = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in cbs]
        refs = [x for x in (info["ref1"], info["ref2"]) if x >= 0] if not info["intra"] else []
        motion = motion_of(results, info, device) if not info["intra"] else None
        dec.decode(pn, info["intra"], refs, info["filter"], q, r["bands"], cbs, motion)
        out[pn] = {"recon": [dec.read(pn, 0, c) for c in range(3)], "coeff": [dec.read(pn, 1, c) for c in range(3)],
                   "output": [dec.read(pn, 9, c) for c in range(3)]}
        if release:
            later = {x for i in infos[k + 1:] if not i["intra"] for x in (i["ref1"], i["ref2"]) if x >= 0}
            for done in [i["pnum"] for i in infos[:k + 1]]:
                if done not in later and done in dec_live(out, dec):
                    dec.release(done)
                    out[done]["released"] = True
    dec.close()
    return out


def dec_live(out, dec):
    return {pn for pn, v in out.items() if not v.get("released")}


def check_round_trip(infos, results, dec):
    for info in infos:
        pn = info["pnum"]
        for c in range(3):
            msg = f"picture {pn} component {c}"
            np.testing.assert_array_equal(dec[pn]["coeff"][c], results[pn]["coeff"][c], err_msg=msg)
            np.testing.assert_array_equal(dec[pn]["recon"][c], results[pn]["recon"][c], err_msg=msg)
            np.testing.assert_array_equal(dec[pn]["output"][c], results[pn]["output"][c], err_msg=msg)


@pytest.mark.parametrize("case", ENCODE_CASES, ids=[c[0] for c in ENCODE_CASES])
def test_decoder_round_trip_matches_reference(gpu, golden, case):
    cfg, infos, results = encoded(gpu, case)
    assert all(i["filter"] in (cfg["intra_filter"], cfg["inter_filter"]) for i in infos)
    dec = decode_all(cfg, infos, results)
    check_round_trip(infos, results, dec)
    crc = np.array([[zlib.crc32(np.ascontiguousarray(dec[i]["output"][c]).tobytes()) for c in range(3)]
                    for i in range(len(infos))], np.uint32)
    np.testing.assert_array_equal(crc, golden("decode.npz")[case[0] + "_crc"])   # the reference decoder's


def test_decoder_device_inputs(gpu):
    cfg, infos, results = encoded(gpu, ENCODE_CASES[1])
    check_round_trip(infos, results, decode_all(cfg, infos, results, device=True))


@pytest.mark.parametrize("device", [False, True], ids=["host", "device"])
def test_decoder_int16_indices(gpu, device):
    """int16 indices (index_bits 16), from host or device memory, decode to the same
    pictures as the int32 ones."""
    cfg, infos, results = encoded(gpu, ENCODE_CASES[1])
    check_round_trip(infos, results, decode_all(cfg, infos, results, device=device, idx16=True))


def test_decoder_rejects_bad_index_bits(gpu):
    from dirac_b200._lib import DgpuError
    from dirac_b200.decoder import SequenceDecoder, decoder_params

    cfg, infos, results = encoded(gpu, ENCODE_CASES[1])
    dec = SequenceDecoder(decoder_params(cfg), max_pictures=2)
    info = infos[0]
    r = results[info["pnum"]]
    q = [r["qindex"][c].reshape(s) for c, s in enumerate(padded_shapes(cfg))]
    I, keep = dec.prepare(info["pnum"], 1, [], info["filter"], q, r["bands"], r["cb_skip"])
    I.index_bits = 8
    with pytest.raises(DgpuError):
        dec.decode_prepared((I, keep))
    I.index_bits = 32
    dec.decode_prepared((I, keep))
    dec.close()


@pytest.mark.parametrize("cformat,depth", [(1, 10), (0, 8), (2, 12)])
def test_decoder_formats_against_oracle(gpu, oracle, cformat, depth):
    """Device decode of 4:2:2 / 4:4:4 / 4:2:0 at 8-12 bits against the oracle's decoder."""
    from dirac_b200 import quant, synth
    from oracle_decoder import decode_picture

    w, h, n = 128, 96, 7
    chroma = {0: "444", 1: "422", 2: "420"}[cformat]
    seq = synth.make_sequence(w, h, n, n_rects=4, vmax=4, seed=40 + cformat, bit_depth=depth, chroma=chroma)
    cfg = dict(cformat=cformat, width=w, height=h, luma_depth=depth, chroma_depth=depth, qf=6.0, l1_sep=3, num_l1=1,
               cpd=20.0, xblen=12, yblen=12, xbsep=8, ybsep=8, mv_precision=2, intra_filter=1, inter_filter=4,
               wlt_depth=3)
    cfg, infos, results = encoded(gpu, cfg=cfg, seq=seq)
    dec = decode_all(cfg, infos, results)
    check_round_trip(infos, results, dec)
    ncb = quant.code_blocks(cfg["wlt_depth"], w, h)
    got = {}
    for info in infos:
        pn = info["pnum"]
        r = results[pn]
        shapes = padded_shapes(cfg)
        b = [r["bands"][c].reshape(-1, 3) for c in range(3)]
        pic = {"intra": info["intra"], "filter": info["filter"],
               "qindex": [r["qindex"][c].reshape(shapes[c]) for c in range(3)],
               "qidx": [x[:, 0] for x in b], "skip": [x[:, 1] for x in b], "cb_skip": r["cb_skip"],
               "me": None if info["intra"] else {k: v for k, v in motion_of(results, info).items()}}
        refs = [got[x] for x in (info["ref1"], info["ref2"]) if x >= 0] if not info["intra"] else None
        got[pn] = decode_picture(cfg, pic, refs, ncb, oracle)
        for c in range(3):
            np.testing.assert_array_equal(dec[pn]["recon"][c], got[pn][c].ravel(), err_msg=f"picture {pn} comp {c}")


@pytest.mark.parametrize("intra", [1, 0])
def test_dequantise_stage_against_oracle(gpu, oracle, intra):
    import torch

    from dirac_b200 import quant
    from dirac_b200.decoder import dequantise

    rng = np.random.default_rng(5 + intra)
    # 77 bands: more than one launch's band table
    comps = [(176, 144, 4), (96, 80, 4), (96, 64, 5), (40, 24, 3), (2, 2, 1), (352, 288, 2), (64, 48, 4)]
    q, bands, ncbs, cbs, want = [], [], [], [], []
    for cw, ch, d in comps:
        nb = 3 * d + 1
        qi = rng.integers(-40, 41, size=(ch, cw), dtype=np.int32)
        qi[rng.random((ch, cw)) < 0.5] = 0
        qidx = rng.integers(0, 60, size=nb).astype(np.int32)
        qidx[rng.integers(0, nb)] = 119
        skip = (rng.random(nb) < 0.15).astype(np.int32)
        ncb = np.asarray(quant.code_blocks(d, cw, ch), np.int32)
        flags = (rng.random(int((ncb[0::2] * ncb[1::2]).sum())) < 0.2).astype(np.uint8)
        want.append(oracle.dequantise(intra, d, qi, qidx, skip, ncb, flags))
        q.append(torch.from_numpy(qi).cuda())
        bands.append(np.stack([qidx, skip], 1))
        ncbs.append(ncb)
        cbs.append(torch.from_numpy(flags).cuda())
    got = dequantise(intra, [c[2] for c in comps], q, bands, ncbs, cbs)
    torch.cuda.synchronize()
    for k in range(len(comps)):
        np.testing.assert_array_equal(got[k].cpu().numpy(), want[k], err_msg=f"component {k}")
    # int16 indices (dgpu_dequantise_batch16)
    got16 = dequantise(intra, [c[2] for c in comps], [t.to(torch.int16) for t in q], bands, ncbs, cbs)
    torch.cuda.synchronize()
    for k in range(len(comps)):
        np.testing.assert_array_equal(got16[k].cpu().numpy(), want[k], err_msg=f"int16, component {k}")
    # in place
    got2 = dequantise(intra, [c[2] for c in comps], q, bands, ncbs, cbs, out=q)
    torch.cuda.synchronize()
    for k in range(len(comps)):
        np.testing.assert_array_equal(got2[k].cpu().numpy(), want[k], err_msg=f"in place, component {k}")


def test_dequantise_int16_extremes(gpu):
    """The int16 form at the int16 extremes equals the int32 form on the same indices."""
    import torch

    from dirac_b200 import quant
    from dirac_b200.decoder import dequantise

    rng = np.random.default_rng(17)
    cw, ch, d = 128, 96, 4
    nb = 3 * d + 1
    qi = rng.integers(-32768, 32768, size=(ch, cw)).astype(np.int16)
    qi.flat[:4] = [32767, -32768, -32767, 0]
    ncb = np.asarray(quant.code_blocks(d, cw, ch), np.int32)
    flags = torch.from_numpy((rng.random(int((ncb[0::2] * ncb[1::2]).sum())) < 0.2).astype(np.uint8)).cuda()
    bands = [np.stack([rng.integers(0, 40, size=nb).astype(np.int32), np.zeros(nb, np.int32)], 1)]
    for intra in (0, 1):
        a = dequantise(intra, d, [torch.from_numpy(qi.astype(np.int32)).cuda()], bands, [ncb], [flags])
        b = dequantise(intra, d, [torch.from_numpy(qi).cuda()], bands, [ncb], [flags])
        torch.cuda.synchronize()
        np.testing.assert_array_equal(b[0].cpu().numpy(), a[0].cpu().numpy())


def test_dequantise_rejects_bad_quantiser(gpu):
    import torch

    from dirac_b200._lib import DgpuError
    from dirac_b200.decoder import dequantise

    q = [torch.zeros((8, 8), dtype=torch.int32, device="cuda")]
    with pytest.raises(DgpuError):
        dequantise(0, [1], q, [np.array([[120, 0], [0, 0], [0, 0], [0, 0]])], [np.ones(8, np.int32)],
                   [torch.zeros(4, dtype=torch.uint8, device="cuda")])


def test_decoder_buffer_rules(gpu):
    """Pictures dropped as soon as no later picture references them: a 5-slot decoder decodes
    the 13-picture GOP sequence identically; a missing reference and a full buffer are
    refused without touching the decoded pictures."""
    from dirac_b200._lib import DgpuError
    from dirac_b200.decoder import SequenceDecoder, decoder_params

    cfg, infos, results = encoded(gpu, ENCODE_CASES[4])
    check_round_trip(infos, results, decode_all(cfg, infos, results, max_pictures=5, release=True))
    dec = SequenceDecoder(decoder_params(cfg), max_pictures=3)
    shapes = padded_shapes(cfg)

    def decode(info):
        r = results[info["pnum"]]
        refs = [x for x in (info["ref1"], info["ref2"]) if x >= 0] if not info["intra"] else []
        dec.decode(info["pnum"], info["intra"], refs, info["filter"],
                   [r["qindex"][c].reshape(shapes[c]) for c in range(3)], r["bands"], r["cb_skip"],
                   motion_of(results, info) if not info["intra"] else None)

    def refs_of(info):
        return {x for x in (info["ref1"], info["ref2"]) if x >= 0} if not info["intra"] else set()

    first_inter = next(i for i in infos if not i["intra"])
    with pytest.raises(DgpuError):
        decode(first_inter)           # its reference is not in the buffer
    for k in range(3):
        decode(infos[k])
    with pytest.raises(DgpuError):
        decode(infos[3])              # three slots, all taken
    with pytest.raises(DgpuError):
        decode(infos[0])              # already in the buffer
    pn0 = infos[0]["pnum"]
    for c in range(3):
        np.testing.assert_array_equal(dec.read(pn0, 0, c), results[pn0]["recon"][c])
    # drop a picture the next one does not reference, then decode the next one into its slot
    drop = next(i["pnum"] for i in infos[:3] if i["pnum"] not in refs_of(infos[3]))
    dec.release(drop)
    with pytest.raises(DgpuError):
        dec.release(drop)             # no longer in the buffer
    decode(infos[3])
    pn3 = infos[3]["pnum"]
    for c in range(3):
        np.testing.assert_array_equal(dec.read(pn3, 0, c), results[pn3]["recon"][c])
    dec.close()
