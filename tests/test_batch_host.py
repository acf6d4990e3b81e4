"""Host-side checks of the picture batch (no GPU): its device-memory size query accepts the
heterogeneous workload's picture descriptions, counts distinct reference planes once, and
rejects invalid descriptions; the workload's algorithmic-byte model."""
import ctypes

from dirac_b200 import _lib
from dirac_b200.batch import BatchMotion, BatchPicture, _picture


def _pic(**kw):
    d = dict(cformat=2, width=352, height=288, luma_depth=8, chroma_depth=8, filter=1, wlt_depth=4, intra=1, qf=7.0,
             cpd=32.0)
    d.update(kw)
    return d


def _bytes(pics, motion=None):
    lib = _lib.load()
    n = len(pics)
    pa = (BatchPicture * n)(*[_picture(p) for p in pics])
    ma = None
    if motion is not None:
        ma = (BatchMotion * n)()
        for k, m in enumerate(motion):
            if m is None:
                continue
            for c in range(3):
                ma[k].ref1[c] = m[0] + c
                if m[1]:
                    ma[k].ref2[c] = m[1] + c
            ma[k].mv1 = ma[k].mode = ma[k].dc = ma[k].split = 0x1000
            ma[k].mv2 = 0x2000 if m[1] else None
    return lib.dgpu_batch_device_bytes(n, pa, ma)


def test_size_query_of_intra_pictures():
    one = _bytes([_pic()])
    assert one > 0
    two = _bytes([_pic(), _pic(width=720, height=576, filter=6, wlt_depth=5)])
    assert two > one


def test_distinct_reference_planes_counted_once():
    from dirac_b200.hetero import block_params

    bp = block_params(352, 288, (12, 12, 8, 8))
    inter = [_pic(intra=0, bp=bp), _pic(intra=0, bp=bp)]
    shared = _bytes(inter, [(0x10000, 0), (0x10000, 0)])       # both predicted from one reference
    separate = _bytes(inter, [(0x10000, 0), (0x20000, 0)])     # each from its own
    up_planes = 4 * (352 * 288 + 2 * 176 * 144) * 2           # one reference's upconverted planes
    assert separate - shared >= up_planes - 3 * 256


def test_invalid_descriptions_rejected():
    assert _bytes([_pic(cformat=3)]) == 0
    assert _bytes([_pic(luma_depth=16)]) == 0
    assert _bytes([_pic(intra=0)]) == 0  # an inter picture needs its motion data


def test_stage_bytes_model():
    from dirac_b200.hetero import stage_bytes, upconvert_bytes
    from dirac_b200.roofline import dwt_bytes

    p = dict(cformat=2, width=64, height=32, wlt_depth=3, intra=0, is_b=1)
    b = stage_bytes([p])
    samples = 64 * 32 + 2 * 32 * 16
    d = dwt_bytes(64, 32, 3) + 2 * dwt_bytes(32, 16, 3)
    assert b["pre"] == d + samples * (4 + 16)
    assert b["post"] == d + samples * (4 + 16)
    assert b["quant"] == 16 * samples

    class T:
        def __init__(self, ptr, n):
            self.p, self.n = ptr, n

        def data_ptr(self):
            return self.p

        def numel(self):
            return self.n

    refs = [T(1, 10), T(2, 5), T(3, 5)]
    assert upconvert_bytes([{"ref1": refs, "ref2": None}, {"ref1": refs, "ref2": refs}, None]) == 10 * 20
