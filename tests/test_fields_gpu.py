"""Field coding (FieldSequenceCompressor, libdirac_encoder/seq_compress.cpp:697-892) on the
device encoder: each interlaced frame loaded as two fields of half its height (the first the
even rows when the top field comes first, pic_io.cpp:464-530), the fields typed, referenced and
ordered by the field GOP (an I frame's second field predicted from its first), the band
weights' vertical frequencies halved (wavelet_utils.cpp:242-243).  Every field's locally
decoded planes equal the stock reference encoder's in field mode (tests/golden/fields.npz),
with the initial entropy-correction factors and with the stock adaptive ones, for the top field
first and the bottom field first, and through a content switch (cut detection on fields)."""
import os
import sys
import zlib

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import FIELD_CASES, TOP_FIELD_FIRST, field_inputs  # noqa: E402

pytestmark = pytest.mark.gpu


def device_params(cfg):
    p = {k: v for k, v in cfg.items() if k not in ("video_format", "use_vlc")}
    p.update(luma_depth=8, chroma_depth=8, top_field_first=TOP_FIELD_FIRST[cfg["video_format"]])
    return p


def check(name, tag, golden, outputs, intra):
    g = golden("fields.npz")
    want, ptype = g[name + tag + "_crc"], g[name + tag + "_ptype"]
    assert sorted(outputs) == list(range(len(ptype)))
    for f in range(len(ptype)):
        if ptype[f] == -1:  # not returned by the reference's API (the last frame's fields)
            continue
        got = [zlib.crc32(np.ascontiguousarray(p).tobytes()) for p in outputs[f]]
        np.testing.assert_array_equal(got, want[f], err_msg=f"{name}{tag} field {f}")
        if ptype[f] >= 0:
            assert intra[f] == ptype[f], (name, f)


@pytest.mark.parametrize("case", FIELD_CASES, ids=[c[0] for c in FIELD_CASES])
def test_field_coding_matches_reference(gpu, golden, case):
    from dirac_b200 import encoder as E
    from dirac_b200.encoder import SequenceEncoder

    seq, cfg = field_inputs(case)
    enc = SequenceEncoder(device_params(cfg), max_pictures=2 * len(seq))
    for f in seq:
        enc.load(f)
    enc.end_sequence()
    outputs, intra = {}, {}
    while True:
        info = enc.code_next()
        if info is None:
            break
        pn = info["pnum"]
        outputs[pn] = [enc.read(pn, E.OUTPUT, c) for c in range(3)]
        intra[pn] = info["intra"]
        if pn % 2 == 1:
            assert outputs[pn][0].size == (cfg["height"] // 2) * cfg["width"]
    enc.close()
    check(case[0], "", golden, outputs, intra)


@pytest.mark.parametrize("case", FIELD_CASES, ids=[c[0] for c in FIELD_CASES])
def test_field_coding_with_host_coder_matches_stock_reference(gpu, golden, case):
    """The stock encoder's adaptive factors on fields, through the library's kind-pipelined
    coding (dgpu_encoder_code_adaptive)."""
    from dirac_b200 import encoder as E
    from dirac_b200.adaptive import AdaptiveCoder
    from dirac_b200.encoder import SequenceEncoder

    seq, cfg = field_inputs(case)
    p = device_params(cfg)
    enc = SequenceEncoder(p, max_pictures=2 * len(seq))
    for f in seq:
        enc.load(f)
    enc.end_sequence()
    coder = AdaptiveCoder(enc, p)
    infos, _, _ = coder.run_native(max_pictures=2 * len(seq), keep_data=False)
    coder.close()
    outputs = {i["pnum"]: [enc.read(i["pnum"], E.OUTPUT, c) for c in range(3)] for i in infos}
    intra = {i["pnum"]: i["intra"] for i in infos}
    enc.close()
    check(case[0], "_adaptive", golden, outputs, intra)


def test_field_loads_keep_device_tensors_and_host_frames_equal(gpu):
    """A frame loaded from host memory and from a CUDA tensor gives the same two fields."""
    import torch

    from dirac_b200 import encoder as E
    from dirac_b200.encoder import SequenceEncoder

    seq, cfg = field_inputs(FIELD_CASES[1])
    p = device_params(cfg)
    res = []
    for dev in (False, True):
        enc = SequenceEncoder(p, max_pictures=8)
        for f in seq[:2]:
            enc.load([torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in f] if dev else f)
        enc.end_sequence()
        out = []
        while True:
            info = enc.code_next()
            if info is None:
                break
            out.append([enc.read(info["pnum"], E.OUTPUT, c) for c in range(3)])
        enc.close()
        res.append(out)
    assert len(res[0]) == 4
    for a, b in zip(*res):
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
