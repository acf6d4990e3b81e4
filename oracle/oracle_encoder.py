"""TEST INFRASTRUCTURE ONLY: the reference's frame-coding loop restated over the oracle's
stage functions, used to check the CUDA sequence encoder picture by picture.

Follows SequenceCompressor::CompressNextPicture (libdirac_encoder/seq_compress.cpp:194-499)
with FrameSequenceCompressor::SetPicTypeAndRefs / CodedToDisplay (seq_compress.cpp:563-686)
and CanEncode (seq_compress.cpp:151-192), and the PictureCompressor steps it calls
(picture_compress.cpp:208-320 motion estimation and intra analysis, 359-472 transform and
residue coding, 532-580 GetCompLambda), with the lambdas of EncoderParams::CalcLambdas
(common.cpp:451-476) and the initial EntropyCorrector factors (common.cpp:79-131), which a
coding loop without the arithmetic coder keeps.  Rate control, prefiltering, field coding
and the bitstream are not part of it.

Band weights and code-block counts come from the library's host helpers, which the oracle
tests pin separately against the reference's own values.
"""
import ctypes
import ctypes.util
import math

import numpy as np

from oracle import BlockParams, Oracle

INTRA_MODE = 0


def cmod(a, b):
    """C++ remainder (truncating toward zero)."""
    r = abs(a) % abs(b)
    return -r if a < 0 else r


def f32(x):
    return float(np.float32(x))


_libm = ctypes.CDLL(ctypes.util.find_library("m"))
_libm.log10f.restype = ctypes.c_float
_libm.log10f.argtypes = [ctypes.c_float]
_libm.sqrtf.restype = ctypes.c_float
_libm.sqrtf.argtypes = [ctypes.c_float]


def log10f(x):
    """std::log10 of a float argument: the C library's single-precision log10."""
    return float(_libm.log10f(x))


def lambdas(qf):
    """EncoderParams::CalcLambdas with its float members."""
    i = f32(math.pow(10.0, (12.0 - f32(qf)) / 2.5) / 16.0)
    l1 = f32(i * 4.0)
    l2 = f32(i * 32.0)
    me = f32(float(_libm.sqrtf(l1)) * 2.0)  # std::sqrt of a float member
    return i, l1, l2, me


def initial_ecf(depth, intra):
    """EntropyCorrector::Init: factors by band (1-based band b at index b-1)."""
    nb = 3 * depth + 1
    out = np.full(nb, 0.75, np.float32)
    out[nb - 4:nb - 1] = 0.85 if intra else 0.75
    out[nb - 1] = 1.0 if intra else 0.85
    return out


class Pic:
    def __init__(self, pnum, planes):
        self.pnum = pnum
        self.orig = [p.copy() for p in planes]
        self.data = [p.copy() for p in planes]
        self.typed = False
        self.intra = True
        self.is_ref = True
        self.refs = []
        self.coded = False
        self.cut = False
        self.me = None
        self.me_refs = None
        self.ratio = 0.0
        self.result = None

    def is_b(self):
        r = self.refs
        return len(r) == 2 and ((r[0] < self.pnum < r[1]) or (r[1] < self.pnum < r[0]))


class OracleEncoder:
    """cfg keys: cformat, width, height, luma_depth, chroma_depth, qf, l1_sep, num_l1, cpd,
    xblen, yblen, xbsep, ybsep, mv_precision, intra_filter, inter_filter, wlt_depth."""

    def __init__(self, cfg, weights_fn, blocks_fn, oracle=None, ecf_fn=None):
        self.cfg = dict(cfg)
        self.ecf_fn = ecf_fn
        self.orc = oracle or Oracle()
        self.weights_fn = weights_fn
        self.blocks_fn = blocks_fn
        c = self.cfg
        self.L1Sep = c["l1_sep"] if c["num_l1"] > 0 else 0
        if c["num_l1"] < 0:
            raise ValueError("num_l1 < 0 is not supported")
        self.num_L1 = c["num_l1"]
        self.gop_len = (self.num_L1 + 1) * self.L1Sep if self.num_L1 > 0 else 10
        self.m_L1_sep = self.L1Sep
        self.gop_start = 0
        self.code = 0
        self.last_read = -1
        self.eos = False
        self.pics = {}
        self.lam_i, self.lam_l1, self.lam_l2, self.lam_me = lambdas(c["qf"])
        w, h = c["width"], c["height"]
        xbsep, ybsep = c["xbsep"], c["ybsep"]
        self.bp = BlockParams(c["mv_precision"], c["xblen"], c["yblen"], xbsep, ybsep,
                              (w + 4 * xbsep - 1) // (4 * xbsep), (h + 4 * ybsep - 1) // (4 * ybsep))
        self.order = []

    # ---- input ----
    def load(self, planes):
        self.last_read += 1
        self.pics[self.last_read] = Pic(self.last_read, planes)

    def end_sequence(self):
        self.eos = True

    # ---- GOP structure ----
    def coded_to_display(self, cnum):
        s = self.m_L1_sep
        if s > 0:
            if cnum == 0:
                return 0
            if cmod(cnum - 1, s) == 0:
                return cnum + s - 1
            return cnum - 1
        return cnum

    def can_encode(self):
        if self.eos:
            if self.num_L1 > 0:
                if self.last_read >= self.code + cmod(self.last_read, self.L1Sep):
                    return True
                if self.code <= self.last_read:
                    self.cur = self.code
                    return True
                return False
            return self.last_read >= self.cur
        return self.last_read >= self.cur + max(4, 2 * self.L1Sep)

    def set_type(self, p):
        pnum = p.pnum
        rel = pnum - self.gop_start
        p.refs = []
        if self.num_L1 > 0:
            s = self.m_L1_sep
            if cmod(rel, self.gop_len) == 0:
                p.intra, p.is_ref = True, self.gop_len > 1
            elif cmod(rel, s) == 0:
                p.intra, p.is_ref = False, True
                p.refs.append(pnum - s)
                if cmod(rel - s, self.gop_len) > 0 and s > 1:
                    p.refs.append(pnum - 2 * s)
            elif cmod(rel + 1, s) == 0:
                p.intra, p.is_ref = False, False
                p.refs.append(pnum - 1)
                if pnum + 1 <= self.last_read:
                    p.refs.append(pnum + 1)
            else:
                p.intra, p.is_ref = False, True
                p.refs.append(pnum - 1)
                nxt = (pnum // s + 1) * s
                if nxt <= self.last_read:
                    p.refs.append(nxt)
        else:
            p.intra, p.is_ref = True, False
        p.typed = True

    # ---- motion estimation (originals only) ----
    def estimate(self, p):
        if p.me is not None and p.me_refs == tuple(p.refs):
            return
        r = [self.pics[k] for k in p.refs]
        c = self.cfg
        p.me = self.orc.motion_estimate(c["cformat"], p.orig, r[0].orig, r[1].orig if len(r) > 1 else None, self.bp,
                                        self.lam_me, 3, c["luma_depth"])
        p.me_refs = tuple(p.refs)
        p.ratio = float(np.count_nonzero(p.me["mode"] == INTRA_MODE)) / float(p.me["mode"].size)

    # ---- one picture ----
    def code_next(self):
        """Codes the next picture in coding order; returns its Pic, or None when more input
        (or the end of the sequence) is needed."""
        if self.L1Sep != self.m_L1_sep and self.L1Sep > 0 and cmod(self.code - 1, self.L1Sep) == 0:
            self.m_L1_sep = self.L1Sep
        self.cur = self.coded_to_display(self.code)
        if not self.can_encode():
            return None
        for pnum in sorted(self.pics):
            q = self.pics[pnum]
            if not q.typed and not q.coded and (self.num_L1 == 0 or pnum < self.cur + self.L1Sep):
                self.set_type(q)
        p = self.pics[self.cur]
        if not p.intra:
            while True:
                self.estimate(p)
                if self.m_L1_sep > 1 and p.ratio > 0.25 and cmod(self.cur, self.L1Sep) == 0:
                    self.m_L1_sep = 1
                    for i in range(self.L1Sep):
                        self.set_type(self.pics[self.cur - i])
                    p.me = None
                    self.cur = self.coded_to_display(self.code)
                    p = self.pics[self.cur]
                    continue
                break
            if p.ratio > 0.3333:
                p.cut = True
                if self.L1Sep > 1 and cmod(self.cur, self.L1Sep) == 0:
                    self.gop_start = p.pnum
                p.intra = True
            else:
                self.motion_compensate(p, 1)
        self.code_residue(p)
        p.coded = True
        p.coded_num = self.code
        self.order.append(p.pnum)
        self.code += 1
        return p

    def motion_compensate(self, p, add_or_sub, clip=False):
        c = self.cfg
        r = [self.pics[k] for k in p.refs]
        me = p.me
        mv2 = me["mv"][1] if len(r) > 1 else None
        p.data = self.orc.motion_compensate(add_or_sub, c["cformat"], p.data, r[0].data,
                                            r[1].data if len(r) > 1 else None, self.bp, me["mv"][0], mv2,
                                            me["mode"], me["dc"], me["split"], c["luma_depth"], c["chroma_depth"])

    def comp_lambda(self, p, comp):
        if p.intra:
            lam = self.lam_i
        else:
            ir = f32(p.ratio)
            lp = self.lam_l2 if p.is_b() else self.lam_l1
            # std::log10 of the float lambdas is the single-precision log10; pow is double
            lam = f32(math.pow(10.0, 3.0 * ir * log10f(self.lam_i) + (1.0 - 3.0 * ir) * log10f(lp)))
        if comp == 1:
            lam = f32(np.float32(lam) * np.float32(1.5))
        elif comp == 2:
            lam = f32(np.float32(lam) * np.float32(0.75))
        return lam

    def code_residue(self, p):
        c = self.cfg
        depth = c["wlt_depth"]
        filt = c["intra_filter"] if p.intra else c["inter_filter"]
        if p.intra:
            cpd_scale = 1.0
        else:
            ir = f32(p.ratio)
            cpd_scale = max(0.125, min(1.2, 5.0 * ir * 1.0 + (1.0 - 5.0 * ir) * 0.125))
        ncb = self.blocks_fn(depth, c["width"], c["height"])
        given = self.ecf_fn(p) if self.ecf_fn is not None else None
        res = {"coeff": [], "qidx": [], "skip": [], "bits": [], "cb_skip": [], "qindex": [], "lambda": [],
               "cpd_scale": cpd_scale, "filter": filt}
        for comp in range(3):
            pic = p.data[comp]
            h, w = pic.shape
            coeff = self.orc.dwt_forward(filt, depth, pic)
            ch, cw = coeff.shape
            wt = self.weights_fn(filt, depth, cw, ch, comp, c["cformat"], c["cpd"], cpd_scale).astype(np.float32)
            lam = self.comp_lambda(p, comp)
            ecf = initial_ecf(depth, p.intra) if given is None else np.asarray(given[comp], np.float32)
            recon, q, sk, bits, cbs, qo = self.orc.code_residue(int(p.intra), depth, coeff, lam, wt, ecf, ncb)
            p.data[comp] = self.orc.dwt_backward(filt, depth, recon, w, h)
            for k, v in (("coeff", recon), ("qidx", q), ("skip", sk), ("bits", bits), ("cb_skip", cbs),
                         ("qindex", qo), ("lambda", lam)):
                res[k].append(v)
        if not p.intra:
            self.motion_compensate(p, 0)
        for comp in range(3):
            self.orc.clip(p.data[comp], c["luma_depth"] if comp == 0 else c["chroma_depth"])
        p.result = res


def encode_sequence(cfg, frames, weights_fn, blocks_fn, oracle=None, ecf_fn=None):
    """Encode a list of frames [(Y, U, V) int16 codec-domain planes]; returns the
    OracleEncoder (pictures in .pics, coding order in .order).  ecf_fn(pic), when given,
    returns the [3][3*depth+1] entropy-correction factors to use for that picture."""
    enc = OracleEncoder(cfg, weights_fn, blocks_fn, oracle, ecf_fn)
    for f in frames:
        enc.load(f)
    enc.end_sequence()
    while enc.code_next() is not None:
        pass
    return enc


def code_picture(pic, planes, weights_fn, blocks_fn, oracle=None, refs=None, me=None):
    """One picture coded as the loop above codes it once its motion data is known (the
    PictureCompressor steps after motion estimation: motion compensation SUBTRACT, transform,
    residue coding, inverse transform, motion compensation ADD and clip).

    pic: the picture's parameters (cformat, width, height, luma_depth, chroma_depth, filter,
    wlt_depth, intra, is_b, qf, cpd, intra_ratio; inter pictures also mv_precision, xblen,
    yblen, xbsep, ybsep); planes: its int16 codec samples; refs: the references' planes (one
    or two); me: the motion data {"mv": [mv1, mv2], "mode", "dc", "split"}.  A B picture
    (is_b) needs two references.  Returns (reconstructed planes, result dict of code_residue)."""
    cfg = {k: pic[k] for k in ("cformat", "width", "height", "luma_depth", "chroma_depth", "qf", "cpd",
                               "wlt_depth")}
    cfg.update(intra_filter=pic["filter"], inter_filter=pic["filter"], l1_sep=1, num_l1=0)
    for k in ("mv_precision", "xblen", "yblen", "xbsep", "ybsep"):
        cfg[k] = pic.get(k, 8 if k != "mv_precision" else 2)
    enc = OracleEncoder(cfg, weights_fn, blocks_fn, oracle)
    pn = 10
    p = Pic(pn, planes)
    p.intra = bool(pic["intra"])
    if not p.intra:
        nref = len(refs)
        if pic.get("is_b") and nref != 2:
            raise ValueError("a B picture has two references")
        ids = [pn - 1, pn + 1] if pic.get("is_b") else [pn - 1, pn - 2][:nref]
        for i, r in zip(ids, refs):
            enc.pics[i] = Pic(i, r)
        p.refs = ids
        p.ratio = pic["intra_ratio"]
        p.me = me
        enc.motion_compensate(p, 1)
    enc.code_residue(p)
    return p.data, p.result
