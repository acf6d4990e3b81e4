"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracles built by oracle/Makefile.

``Oracle`` wraps liboracle.so, this project's plain-C restatement of the Dirac hot path
(oracle/dirac_oracle.c).  ``Reference`` wraps oracle/_ref/libdirac_ref.so, the reference
codec's own C++ compiled from its sources plus the stage driver oracle/ref_driver.cpp; it
exists only where the reference sources were available at build time.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use this module.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libdirac_ref.so")
# the reference with its hot-path method bodies calling libdiracgpu (oracle/dropin/)
DROPIN_SO = os.path.join(HERE, "_ref", "libdirac_dropin.so")


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class BlockParams(ctypes.Structure):
    """orc_block_params / RefBlockDesc: precision, xblen, yblen, xbsep, ybsep, xnum_sb, ynum_sb."""

    _fields_ = [(n, ctypes.c_int) for n in
                ("precision", "xblen", "yblen", "xbsep", "ybsep", "xnum_sb", "ynum_sb")]


def chroma_shift(cformat):
    """(xshift, yshift) of the chroma planes for ChromaFormat 0 (444), 1 (422), 2 (420)."""
    return {0: (0, 0), 1: (1, 0), 2: (1, 1)}[cformat]


def _ptrs(arrs):
    return (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def _mc_args(mv1, mv2, mode, dc, split):
    mv1 = np.ascontiguousarray(mv1, dtype=np.int16)
    mv2 = np.ascontiguousarray(mv2 if mv2 is not None else mv1, dtype=np.int16)
    mode = np.ascontiguousarray(mode, dtype=np.uint8)
    dc = np.ascontiguousarray(dc, dtype=np.int16)
    split = np.ascontiguousarray(split, dtype=np.uint8)
    return mv1, mv2, mode, dc, split


def padded(w, h, depth):
    mul = 1 << depth
    return (w + mul - 1) // mul * mul, (h + mul - 1) // mul * mul


class Oracle:
    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle oracle`")
        self.lib = ctypes.CDLL(path)

    def clip(self, pic, bit_depth):
        """Picture::ClipComponent, in place on a contiguous int16 array."""
        assert pic.dtype == np.int16 and pic.flags["C_CONTIGUOUS"]
        self.lib.orc_clip(_p(pic), ctypes.c_size_t(pic.size), ctypes.c_int(bit_depth))
        return pic

    def dwt_min_len(self, filt):
        return self.lib.orc_dwt_min_len(filt)

    def rect_lp_filter(self, pic, qf, strength):
        """LPFilter (RECTLP) of a 2-D int16 component; returns the filtered copy."""
        p = np.array(pic, dtype=np.int16, copy=True, order="C")
        h, w = p.shape
        if self.lib.orc_rect_lp_filter(_p(p), w, h, ctypes.c_float(qf), strength):
            raise ValueError("orc_rect_lp_filter failed")
        return p

    def diag_lp_filter(self, pic, qf, strength):
        """DiagFilter (DIAGLP) of a 2-D int16 component; returns the filtered copy."""
        p = np.array(pic, dtype=np.int16, copy=True, order="C")
        h, w = p.shape
        if self.lib.orc_diag_lp_filter(_p(p), w, h, ctypes.c_float(qf), strength):
            raise ValueError("orc_diag_lp_filter failed")
        return p

    def cwm_filter(self, pic, strength):
        """CWMFilterComponent of a 2-D int16 component; returns the filtered copy."""
        p = np.ascontiguousarray(pic, dtype=np.int16)
        out = np.empty_like(p)
        h, w = p.shape
        if self.lib.orc_cwm_filter(_p(p), _p(out), w, h, strength):
            raise ValueError("orc_cwm_filter failed")
        return out

    def dwt_forward(self, filt, depth, pic, cw=None, ch=None):
        pic = np.ascontiguousarray(pic, dtype=np.int16)
        h, w = pic.shape
        if cw is None:
            cw, ch = padded(w, h, depth)
        coeff = np.zeros((ch, cw), np.int32)
        rc = self.lib.orc_dwt_forward(filt, depth, _p(pic), w, h, w, _p(coeff), cw, ch, cw)
        if rc:
            raise ValueError(f"orc_dwt_forward rc={rc}")
        return coeff

    def dwt_backward(self, filt, depth, coeff, w, h):
        c = np.array(coeff, dtype=np.int32, copy=True, order="C")
        ch, cw = c.shape
        pic = np.zeros((h, w), np.int16)
        rc = self.lib.orc_dwt_backward(filt, depth, _p(c), cw, ch, cw, _p(pic), w, h, w)
        if rc:
            raise ValueError(f"orc_dwt_backward rc={rc}")
        return pic

    def upconvert(self, pic, bit_depth):
        pic = np.ascontiguousarray(pic, dtype=np.int16)
        h, w = pic.shape
        up = np.zeros((2 * h, 2 * w), np.int16)
        rc = self.lib.orc_upconvert(_p(pic), w, h, w, bit_depth, _p(up), 2 * w)
        if rc:
            raise ValueError(f"orc_upconvert rc={rc}")
        return up

    def downconvert(self, pic):
        pic = np.ascontiguousarray(pic, dtype=np.int16)
        h, w = pic.shape
        out = np.zeros((h // 2, w // 2), np.int16)
        rc = self.lib.orc_downconvert(_p(pic), w, h, w, _p(out), w // 2)
        if rc:
            raise ValueError(f"orc_downconvert rc={rc}")
        return out


    def motion_compensate(self, add_or_sub, cformat, pic, ref1, ref2, bp, mv1, mv2, mode, dc, split,
                          luma_depth=8, chroma_depth=8, weights=(1, 1, 1)):
        """OBMC of a 3-component picture; refs are plain pictures (upconverted here).  weights:
        the reference picture weights (ref1, ref2, precision bits)."""
        out = [np.array(p, dtype=np.int16, copy=True, order="C") for p in pic]
        r2 = ref2 if ref2 is not None else ref1
        up1 = [self.upconvert(r, luma_depth if c == 0 else chroma_depth) for c, r in enumerate(ref1)]
        up2 = [self.upconvert(r, luma_depth if c == 0 else chroma_depth) for c, r in enumerate(r2)]
        mv1, mv2, mode, dc, split = _mc_args(mv1, mv2, mode, dc, split)
        h, w = out[0].shape
        rc = self.lib.orc_motion_compensate_wt(add_or_sub, cformat, w, h, ctypes.byref(bp), _p(mv1), _p(mv2),
                                               _p(mode), _p(dc), _p(split), _ptrs(out), _ptrs(up1), _ptrs(up2),
                                               *[int(x) for x in weights])
        if rc:
            raise ValueError(f"orc_motion_compensate rc={rc}")
        return out


    def motion_estimate(self, cformat, pic, ref1, ref2, bp, lambda_, stages=3, luma_depth=8):
        return _me_call(self.lib.orc_motion_estimate, True, cformat, pic, ref1, ref2, bp, lambda_, stages,
                        luma_depth)

    def me_depth(self, w, h):
        return self.lib.orc_me_depth(w, h)

    def code_residue(self, intra, depth, coeff, lambda_, band_wt, band_ecf, band_ncb):
        """Quantiser choice + quantisation; returns (recon, qidx, skip, bits, cb_skip, qindices)."""
        c = np.array(coeff, dtype=np.int32, copy=True, order="C")
        ch, cw = c.shape
        nb = 3 * depth + 1
        wt = np.ascontiguousarray(band_wt, dtype=np.float32)
        ecf = np.ascontiguousarray(band_ecf, dtype=np.float32)
        ncb = np.ascontiguousarray(band_ncb, dtype=np.int32)
        q = np.zeros(nb, np.int32)
        sk = np.zeros(nb, np.int32)
        bits = np.zeros(nb, np.int32)
        cbs = np.zeros(int(np.sum(ncb[0::2] * ncb[1::2])), np.uint8)
        qo = np.zeros_like(c)
        rc = self.lib.orc_code_residue(intra, depth, _p(c), cw, ch, ctypes.c_float(lambda_), _p(wt), _p(ecf), _p(ncb),
                                       _p(q), _p(sk), _p(bits), _p(cbs), _p(qo))
        if rc:
            raise ValueError(f"orc_code_residue rc={rc}")
        return c, q, sk, bits, cbs, qo

    def dequantise(self, intra, depth, qindex, band_qidx, band_skip, band_ncb, cb_skip):
        """The decoder's dequantisation of one component; returns the coefficients."""
        q = np.ascontiguousarray(qindex, dtype=np.int32)
        ch, cw = q.shape
        out = np.zeros_like(q)
        bq = np.ascontiguousarray(band_qidx, dtype=np.int32)
        bs = np.ascontiguousarray(band_skip, dtype=np.int32)
        ncb = np.ascontiguousarray(band_ncb, dtype=np.int32)
        cbs = np.ascontiguousarray(cb_skip, dtype=np.uint8)
        rc = self.lib.orc_dequantise(int(intra), depth, _p(q), _p(out), cw, ch, _p(ncb), _p(bq), _p(bs), _p(cbs))
        if rc:
            raise ValueError(f"orc_dequantise rc={rc}")
        return out


def _me_call(fn, is_oracle, cformat, pic, ref1, ref2, bp, lambda_, stages, luma_depth):
    """Shared driver of orc_motion_estimate / ref_motion_estimate; returns a dict of arrays."""
    nref = 2 if ref2 is not None else 1
    pic = [np.ascontiguousarray(p, dtype=np.int16) for p in pic]
    r1 = [np.ascontiguousarray(p, dtype=np.int16) for p in ref1]
    r2 = [np.ascontiguousarray(p, dtype=np.int16) for p in (ref2 if ref2 is not None else ref1)]
    h, w = pic[0].shape
    nsb = bp.xnum_sb * bp.ynum_sb
    nb = 16 * nsb
    mv = np.zeros((nref, nb, 2), np.int16)
    cost = np.zeros((nref, nb, 3), np.float32)
    mode = np.zeros(nb, np.uint8)
    dc = np.zeros((3, nb), np.int16)
    split = np.zeros(nsb, np.uint8)
    sbcost = np.zeros(nsb, np.float32)
    if is_oracle:
        rc = fn(cformat, w, h, ctypes.byref(bp), nref, _ptrs(pic), _ptrs(r1), _ptrs(r2), luma_depth,
                ctypes.c_float(lambda_), stages, _p(mv), _p(cost), _p(mode), _p(dc), _p(split), _p(sbcost))
    else:
        rc = fn(cformat, w, h, luma_depth, luma_depth, ctypes.byref(bp), nref, _ptrs(pic), _ptrs(r1), _ptrs(r2),
                ctypes.c_float(lambda_), stages, _p(mv), _p(cost), _p(mode), _p(dc), _p(split), _p(sbcost))
    if rc:
        raise ValueError(f"motion estimation failed rc={rc}")
    ynb, xnb = 4 * bp.ynum_sb, 4 * bp.xnum_sb
    return {"mv": mv.reshape(nref, ynb, xnb, 2), "cost": cost.reshape(nref, ynb, xnb, 3),
            "mode": mode.reshape(ynb, xnb), "dc": dc.reshape(3, ynb, xnb),
            "split": split.reshape(bp.ynum_sb, bp.xnum_sb), "sbcost": sbcost.reshape(bp.ynum_sb, bp.xnum_sb)}


class Reference:
    """The reference codec itself (plain-C build), driven stage by stage."""

    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle` where the reference sources exist")
        self.lib = ctypes.CDLL(path)

    @staticmethod
    def available(path=REF_SO):
        return os.path.exists(path)

    def dwt_forward(self, filt, depth, pic, cw=None, ch=None):
        pic = np.ascontiguousarray(pic, dtype=np.int16)
        h, w = pic.shape
        if cw is None:
            cw, ch = padded(w, h, depth)
        coeff = np.zeros((ch, cw), np.int32)
        if self.lib.ref_dwt_forward(filt, depth, _p(pic), w, h, _p(coeff), cw, ch):
            raise ValueError("ref_dwt_forward failed")
        return coeff

    def dwt_backward(self, filt, depth, coeff, w, h):
        c = np.array(coeff, dtype=np.int32, copy=True, order="C")
        ch, cw = c.shape
        pic = np.zeros((h, w), np.int16)
        if self.lib.ref_dwt_backward(filt, depth, _p(c), cw, ch, _p(pic), w, h):
            raise ValueError("ref_dwt_backward failed")
        return pic

    def upconvert(self, pic, bit_depth):
        pic = np.ascontiguousarray(pic, dtype=np.int16)
        h, w = pic.shape
        up = np.zeros((2 * h, 2 * w), np.int16)
        if self.lib.ref_upconvert(_p(pic), w, h, bit_depth, _p(up)):
            raise ValueError("ref_upconvert failed")
        return up

    def rect_lp_filter(self, pic, qf, strength):
        p = np.array(pic, dtype=np.int16, copy=True, order="C")
        h, w = p.shape
        if self.lib.ref_lp_filter(_p(p), w, h, ctypes.c_float(qf), strength):
            raise ValueError("ref_lp_filter failed")
        return p

    def diag_lp_filter(self, pic, qf, strength):
        p = np.array(pic, dtype=np.int16, copy=True, order="C")
        h, w = p.shape
        if self.lib.ref_diag_filter(_p(p), w, h, ctypes.c_float(qf), strength):
            raise ValueError("ref_diag_filter failed")
        return p

    def cwm_filter(self, pic, strength):
        p = np.array(pic, dtype=np.int16, copy=True, order="C")
        h, w = p.shape
        if self.lib.ref_cwm_filter(_p(p), w, h, strength):
            raise ValueError("ref_cwm_filter failed")
        return p

    def downconvert(self, pic):
        pic = np.ascontiguousarray(pic, dtype=np.int16)
        h, w = pic.shape
        out = np.zeros((h // 2, w // 2), np.int16)
        if self.lib.ref_downconvert(_p(pic), w, h, _p(out)):
            raise ValueError("ref_downconvert failed")
        return out

    def motion_compensate(self, add_or_sub, cformat, pic, ref1, ref2, bp, mv1, mv2, mode, dc, split,
                          luma_depth=8, chroma_depth=8, weights=(1, 1, 1)):
        out = [np.array(p, dtype=np.int16, copy=True, order="C") for p in pic]
        nref = 2 if ref2 is not None else 1
        r1 = [np.ascontiguousarray(r, dtype=np.int16) for r in ref1]
        r2 = [np.ascontiguousarray(r, dtype=np.int16) for r in (ref2 if ref2 is not None else ref1)]
        mv1, mv2, mode, dc, split = _mc_args(mv1, mv2, mode, dc, split)
        h, w = out[0].shape
        rc = self.lib.ref_motion_compensate_wt(add_or_sub, cformat, w, h, luma_depth, chroma_depth,
                                               ctypes.byref(bp), nref, _p(mv1), _p(mv2), _p(mode), _p(dc),
                                               _p(split), _ptrs(out), _ptrs(r1), _ptrs(r2), *[int(x) for x in weights])
        if rc:
            raise ValueError("ref_motion_compensate failed")
        return out

    def motion_estimate(self, cformat, pic, ref1, ref2, bp, lambda_, stages=3, luma_depth=8):
        return _me_call(self.lib.ref_motion_estimate, False, cformat, pic, ref1, ref2, bp, lambda_, stages,
                        luma_depth)

    def code_residue(self, cformat, w, h, comp, intra, filt, depth, coeff, lambda_, cpd_scale=1.0):
        """The reference's residue coding of one component; returns a dict with the
        reconstruction and the per-band / per-code-block choices and their inputs."""
        c = np.array(coeff, dtype=np.int32, copy=True, order="C")
        ch, cw = c.shape
        nb = 3 * depth + 1
        q = np.zeros(nb, np.int32)
        sk = np.zeros(nb, np.int32)
        wt = np.zeros(nb, np.float64)
        ecf = np.zeros(nb, np.float32)
        bits = np.zeros(nb, np.int32)
        ncb = np.zeros(2 * nb, np.int32)
        cbs = np.zeros(1 << 20, np.uint8)
        rc = self.lib.ref_code_residue(cformat, w, h, comp, intra, filt, depth, _p(c), cw, ch, ctypes.c_float(lambda_),
                                       ctypes.c_float(cpd_scale), _p(q), _p(sk), _p(wt), _p(ecf), _p(bits), _p(ncb),
                                       _p(cbs))
        if rc:
            raise ValueError("ref_code_residue failed")
        ncbt = int(np.sum(ncb[0::2] * ncb[1::2]))
        return {"recon": c, "qidx": q, "skip": sk, "wt": wt, "ecf": ecf, "bits": bits, "ncb": ncb,
                "cb_skip": cbs[:ncbt].copy()}

    def code_residue_vlc_bytes(self, cformat, w, h, comp, intra, filt, depth, coeff, lambda_, cpd_scale=1.0):
        """As code_residue_bytes with the variable-length band coders (-use_vlc); also
        "compress_bytes": what each coder's Compress returned (whole bytes before alignment)."""
        c = np.array(coeff, dtype=np.int32, copy=True, order="C")
        ch, cw = c.shape
        nb = 3 * depth + 1
        q, sk, bits = np.zeros(nb, np.int32), np.zeros(nb, np.int32), np.zeros(nb, np.int32)
        wt, ecf = np.zeros(nb, np.float64), np.zeros(nb, np.float32)
        ncb = np.zeros(2 * nb, np.int32)
        cbs = np.zeros(1 << 20, np.uint8)
        cap = 8 * c.size + 4096
        data = np.zeros(cap, np.uint8)
        nbytes, whole = np.zeros(nb, np.int32), np.zeros(nb, np.int32)
        rc = self.lib.ref_code_residue_vlc_bytes(cformat, w, h, comp, intra, filt, depth, _p(c), cw, ch,
                                                 ctypes.c_float(lambda_), ctypes.c_float(cpd_scale), _p(q), _p(sk),
                                                 _p(wt), _p(ecf), _p(bits), _p(ncb), _p(cbs), _p(data),
                                                 ctypes.c_longlong(cap), _p(nbytes), _p(whole))
        if rc:
            raise ValueError(f"ref_code_residue_vlc_bytes failed: {rc}")
        ncbt = int(np.sum(ncb[0::2] * ncb[1::2]))
        return {"recon": c, "qidx": q, "skip": sk, "wt": wt, "ecf": ecf, "bits": bits, "ncb": ncb,
                "cb_skip": cbs[:ncbt].copy(), "data": data[:int(nbytes.sum())].copy(), "band_bytes": nbytes,
                "compress_bytes": whole}

    def code_inter_indices_bytes(self, depth, idx, band_ncb):
        """The reference's band coders on given signed indices of an inter component, every
        quantiser at index 0 (factor 1); band_ncb: [nb][2] code blocks across and down.
        Returns (data, band_bytes, cb_skip), data DC band first."""
        q = np.ascontiguousarray(idx, dtype=np.int32)
        ch, cw = q.shape
        nb = 3 * depth + 1
        ncb = np.ascontiguousarray(band_ncb, dtype=np.int32).reshape(-1)
        cbs = np.zeros(int(np.sum(ncb[0::2] * ncb[1::2])), np.uint8)
        cap = 8 * q.size + 4096
        data = np.zeros(cap, np.uint8)
        nbytes = np.zeros(nb, np.int32)
        rc = self.lib.ref_code_inter_indices_bytes(depth, _p(q), cw, ch, _p(ncb), _p(cbs), _p(data),
                                                   ctypes.c_longlong(cap), _p(nbytes))
        if rc:
            raise ValueError(f"ref_code_inter_indices_bytes failed: {rc}")
        return data[:int(nbytes.sum())].copy(), nbytes, cbs

    def code_residue_bytes(self, cformat, w, h, comp, intra, filt, depth, coeff, lambda_, cpd_scale=1.0):
        """As code_residue, plus the reference band coders' output: "data" (every coded band's
        arithmetic-coded bytes, DC band first) and "band_bytes" (per band, 0 when skipped)."""
        c = np.array(coeff, dtype=np.int32, copy=True, order="C")
        ch, cw = c.shape
        nb = 3 * depth + 1
        q = np.zeros(nb, np.int32)
        sk = np.zeros(nb, np.int32)
        wt = np.zeros(nb, np.float64)
        ecf = np.zeros(nb, np.float32)
        bits = np.zeros(nb, np.int32)
        ncb = np.zeros(2 * nb, np.int32)
        cbs = np.zeros(1 << 20, np.uint8)
        cap = 8 * c.size + 4096
        data = np.zeros(cap, np.uint8)
        nbytes = np.zeros(nb, np.int32)
        rc = self.lib.ref_code_residue_bytes(cformat, w, h, comp, intra, filt, depth, _p(c), cw, ch,
                                             ctypes.c_float(lambda_), ctypes.c_float(cpd_scale), _p(q), _p(sk), _p(wt),
                                             _p(ecf), _p(bits), _p(ncb), _p(cbs), _p(data), ctypes.c_longlong(cap),
                                             _p(nbytes))
        if rc:
            raise ValueError(f"ref_code_residue_bytes failed: {rc}")
        ncbt = int(np.sum(ncb[0::2] * ncb[1::2]))
        return {"recon": c, "qidx": q, "skip": sk, "wt": wt, "ecf": ecf, "bits": bits, "ncb": ncb,
                "cb_skip": cbs[:ncbt].copy(), "data": data[:int(nbytes.sum())].copy(), "band_bytes": nbytes}


class RefEncParams(ctypes.Structure):
    """Mirror of RefEncParams in oracle/ref_encoder.cpp."""

    _fields_ = [("video_format", ctypes.c_int), ("cformat", ctypes.c_int), ("width", ctypes.c_int),
                ("height", ctypes.c_int), ("qf", ctypes.c_float), ("l1_sep", ctypes.c_int),
                ("num_l1", ctypes.c_int), ("cpd", ctypes.c_float), ("xblen", ctypes.c_int),
                ("yblen", ctypes.c_int), ("xbsep", ctypes.c_int), ("ybsep", ctypes.c_int),
                ("mv_precision", ctypes.c_int), ("intra_filter", ctypes.c_int), ("inter_filter", ctypes.c_int),
                ("wlt_depth", ctypes.c_int), ("use_vlc", ctypes.c_int), ("field_coding", ctypes.c_int)]


def reference_encode(cfg, frames, freeze=True, path=REF_SO):
    """Encode 8-bit frames [(Y, U, V) uint8 planes] with the reference encoder's public API.
    cfg: dict with the RefEncParams fields.  Returns (recon frames as (Y, U, V) uint8 planes
    by picture number, per-picture intra flags, total bitstream bytes)."""
    lib = Reference(path).lib
    p = RefEncParams(**cfg)
    n = len(frames)
    flat = np.concatenate([np.concatenate([np.ascontiguousarray(c, np.uint8).ravel() for c in f]) for f in frames])
    recon = np.zeros_like(flat)
    fields = bool(cfg.get("field_coding", 0))
    npics = 2 * n if fields else n
    ptype = np.zeros(npics, np.int32)
    nbytes = ctypes.c_longlong(0)
    rc = lib.ref_encode_sequence(ctypes.byref(p), n, _p(flat), int(freeze), _p(recon), _p(ptype), ctypes.byref(nbytes))
    if rc:
        raise ValueError("ref_encode_sequence failed")
    shapes = [(c.shape[0] // 2, c.shape[1]) if fields else c.shape for c in frames[0]]
    return _split_frames(recon, shapes, npics), ptype, nbytes.value


def _split_frames(flat, shapes, n):
    fsize = sum(int(np.prod(s)) for s in shapes)
    out = []
    for i in range(n):
        fr, o = [], i * fsize
        for s in shapes:
            k = int(np.prod(s))
            fr.append(flat[o:o + k].reshape(s))
            o += k
        out.append(tuple(fr))
    return out


def reference_encode_stream(cfg, frames, freeze=True, path=REF_SO):
    """As reference_encode, returning (recon frames, intra flags, the coded bitstream bytes)."""
    lib = Reference(path).lib
    p = RefEncParams(**cfg)
    n = len(frames)
    flat = np.concatenate([np.concatenate([np.ascontiguousarray(c, np.uint8).ravel() for c in f]) for f in frames])
    recon = np.zeros_like(flat)
    ptype = np.zeros(n, np.int32)
    cap = max(1 << 20, 2 * flat.size)
    stream = np.zeros(cap, np.uint8)
    nbytes = ctypes.c_longlong(0)
    rc = lib.ref_encode_stream(ctypes.byref(p), n, _p(flat), int(freeze), _p(recon), _p(ptype), _p(stream),
                               ctypes.c_longlong(cap), ctypes.byref(nbytes))
    if rc:
        raise ValueError(f"ref_encode_stream failed: {rc}")
    return _split_frames(recon, [c.shape for c in frames[0]], n), ptype, stream[:nbytes.value].copy()


def reference_decode(stream, width, height, cformat, nframes, path=REF_SO):
    """Decode an 8-bit Dirac bitstream with the reference decoder's public API; returns the
    frames [(Y, U, V) uint8 planes] by frame number (None where no frame was delivered)."""
    lib = Reference(path).lib
    xs, ys = chroma_shift(cformat)
    cw, ch = width >> xs, height >> ys
    data = np.ascontiguousarray(stream, np.uint8)
    flat = np.zeros(nframes * (width * height + 2 * cw * ch), np.uint8)
    got = np.zeros(nframes, np.int32)
    rc = lib.ref_decode_stream(_p(data), ctypes.c_longlong(data.size), width, height, cw, ch, nframes, _p(flat),
                               _p(got))
    if rc < 0:
        raise ValueError("ref_decode_stream: invalid stream")
    frames = _split_frames(flat, [(height, width), (ch, cw), (ch, cw)], nframes)
    return [f if got[i] else None for i, f in enumerate(frames)]
