"""A sequence coded as the stock reference encoder codes it: the device encoder's pictures,
their subbands arithmetic-coded on host threads and the entropy-correction factors adapted from
the coded byte counts after every component (SequenceCompressor, seq_compress.cpp:194-499;
EntropyCorrector::Update, common.cpp:134-151).

The reference keeps one set of factors per picture kind, intra, B or other inter, and both the
quantiser choice and the update index them by the picture's kind (EntropyCorrector::Factor and
Update, common.cpp:67-78, 138-151).  A picture therefore depends only on the host coding of the
last picture of its own kind, not on the picture coded just before it: in an I P B B P B B ...
coding order most pictures can be finished on the device while the previous one is still being
coded on the host.  AdaptiveCoder runs that pipeline.  Per picture, in coding order: prepare it
on the device (motion estimation, compensation, transform: no factors needed), wait for the
coding of the last picture of its kind, finish it (quantiser choice with the kind's factors,
quantisation, reconstruction), queue the copies of its indices, band and code-block choices and
motion data into page-locked buffers of its kind, and hand it to a coding thread, which waits
for the copies, codes the bands and updates the kind's factors.  The pictures, bands and bytes
equal those of the serial loop (code, adapt, then the next picture)."""
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

from . import _lib
from . import encoder as E
from . import quant
from .entropy import EntropyCorrector, code_bands

# results a bitstream writer needs from a coded picture: the band coder's inputs and the
# motion data (vectors, modes, intra DC values, superblock splitting)
CODED_ITEMS = [(E.QINDEX, c) for c in range(3)] + [(E.BANDS, c) for c in range(3)] + \
              [(E.CBSKIP, c) for c in range(3)] + [(E.MV, 0), (E.MODE, 0), (E.DC, 0), (E.SPLIT, 0)]


def picture_kind(info):
    """EntropyCorrector's index of a picture: 0 intra, 1 B, 2 other inter."""
    return 0 if info["intra"] else (1 if info["is_b"] else 2)


class AdaptiveCoder:
    """Stock-encoder coding of a SequenceEncoder's pictures (arithmetic-coded subbands).

    enc: the SequenceEncoder; params: its parameter dict.  run() codes every picture the encoder
    has input for and returns their infos in coding order; on_finished(info) is called on the
    calling thread after each picture's device coding has been queued (its device results, such
    as DGPU_ENC_OUTPUT, are then readable), on_coded(info, got, data, band_bytes) on a coding
    thread after its bands are coded (got: the copied results by (item, component), valid until
    the next picture of the same kind is read)."""

    def __init__(self, enc, params, threads=3):
        self.enc = enc
        self.lib = _lib.load()
        self.depth = params["wlt_depth"]
        self.ncb = quant.code_blocks(self.depth, enc.shapes[0][1], enc.shapes[0][0])  # picture (field) size
        mul = 1 << self.depth
        self.qshapes = [((h + mul - 1) // mul * mul, (w + mul - 1) // mul * mul) for h, w in enc.shapes]
        self.ex = ThreadPoolExecutor(threads)
        self.bufs = {}
        self.lock = threading.Lock()
        self.ec = None
        self.d2h_bytes = 0
        self.coded_bytes = 0
        self.phases = dict.fromkeys(("prepare", "wait", "finish", "read", "code"), 0.0)

    def close(self):
        self.ex.shutdown(wait=True)

    def run_native(self, max_pictures=None, keep_data=True):
        """The same pipeline in the library (dgpu_encoder_code_adaptive): no Python between the
        pictures, the host coding on the library's threads.  Returns (infos in coding order,
        coded data per picture or None, band bytes [pictures][3][3*depth+1])."""
        import ctypes

        n = max_pictures if max_pictures is not None else 4096
        self.ec = EntropyCorrector(self.depth)
        infos = (E.PictureInfo * n)()
        nb = 3 * self.depth + 1
        bb = np.zeros((n, 3, nb), np.int32)
        total = ctypes.c_size_t(0)
        d2h = ctypes.c_size_t(0)
        npics = ctypes.c_int(0)
        rc = self.lib.dgpu_encoder_code_adaptive(self.enc.handle, self.ec.state.ctypes.data, n, infos, None, 0,
                                                 ctypes.byref(total), bb.ctypes.data, ctypes.byref(d2h),
                                                 ctypes.byref(npics))
        _lib.check(rc, "dgpu_encoder_code_adaptive")
        out = np.empty(total.value if keep_data else 0, np.uint8)
        if keep_data and total.value:
            got = ctypes.c_size_t(0)
            _lib.check(self.lib.dgpu_encoder_adaptive_data(self.enc.handle, out.ctypes.data, out.size,
                                                           ctypes.byref(got)), "dgpu_encoder_adaptive_data")
        k = npics.value
        self.d2h_bytes += d2h.value
        self.coded_bytes += total.value
        bb = bb[:k]
        data = None
        if keep_data:
            data, at = [], 0
            for i in range(k):
                m = int(bb[i].sum())
                data.append(out[at:at + m])
                at += m
        return [infos[i].as_dict() for i in range(k)], data, bb

    def _read(self, info, kind):
        pn = info["pnum"]
        got = {}
        for what, c in CODED_ITEMS:
            n = self.lib.dgpu_encoder_item_bytes(self.enc.handle, pn, what, c)
            if n == 0:
                continue
            b = self.bufs.get((kind, what, c))
            if b is None or b.numel() != n:
                b = self.bufs[(kind, what, c)] = torch.empty(n, dtype=torch.uint8, pin_memory=True)
            _lib.check(self.lib.dgpu_encoder_read(self.enc.handle, pn, what, c, b.data_ptr(), n, 2),
                       "dgpu_encoder_read")
            self.d2h_bytes += n
            got[(what, c)] = b.numpy()
        ev = torch.cuda.Event()
        ev.record(self.enc.stream)
        return got, ev

    def _code(self, info, got, ev, on_coded):
        import time

        ev.synchronize()
        t0 = time.perf_counter()
        q = [got[(E.QINDEX, c)].view(np.int32).reshape(self.qshapes[c]) for c in range(3)]
        bands = [got[(E.BANDS, c)].view(np.int32).reshape(-1, 3) for c in range(3)]
        cbs = [got[(E.CBSKIP, c)] for c in range(3)]
        data, per = code_bands([info["intra"]] * 3, [self.depth] * 3, q, bands, [self.ncb] * 3, cbs)
        for c in range(3):
            self.ec.update(info["intra"], info["is_b"], c, bands[c][:, 1], bands[c][:, 2], per[c])
        with self.lock:
            self.coded_bytes += int(data.size)
            self.phases["code"] += time.perf_counter() - t0
        if on_coded is not None:
            on_coded(info, got, data, per)

    def run(self, on_finished=None, on_coded=None):
        import time

        enc = self.enc
        self.ec = EntropyCorrector(self.depth)
        last = {}
        infos = []
        ph = self.phases
        try:
            while True:
                t0 = time.perf_counter()
                nxt = enc.prepare_next()
                t1 = time.perf_counter()
                ph["prepare"] += t1 - t0
                if nxt is None:
                    break
                kind = picture_kind(nxt)
                if kind in last:
                    last.pop(kind).result()  # the kind's factors are up to date
                t2 = time.perf_counter()
                info = enc.finish_next(ecf_state=self.ec.state)
                t3 = time.perf_counter()
                if on_finished is not None:
                    on_finished(info)
                got, ev = self._read(info, kind)
                t4 = time.perf_counter()
                ph["wait"] += t2 - t1
                ph["finish"] += t3 - t2
                ph["read"] += t4 - t3
                last[kind] = self.ex.submit(self._code, info, got, ev, on_coded)
                infos.append(info)
        finally:
            for f in last.values():
                f.result()
        return infos
