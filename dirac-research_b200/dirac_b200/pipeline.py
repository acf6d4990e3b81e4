"""Device-resident frame pipeline for a sequence of pictures (the bench workload).

A Pipeline owns the device buffers for a batch of frames (int16 component planes,
int32 coefficient arrays, library scratch) and runs the hot-path stages on them through
the C ABI.  Stages implemented so far: forward wavelet transform of every component
(intra filter on frame 0, inter filter on the others), inverse transform back to the
picture planes.
"""
import torch

from . import _lib
from .wavelet import FORWARD, BACKWARD, padded_size

CHROMA = {"420": (2, 2), "422": (2, 1), "444": (1, 1)}


def dwt_algorithmic_bytes(cw, ch, depth, direction):
    """Bytes a transform must move once: level 1 reads int16 picture samples and writes int32
    coefficients (forward; the reverse for the inverse), deeper levels read and write int32 over
    their low-pass region."""
    total = 0
    for lev in range(1, depth + 1):
        n = (cw >> (lev - 1)) * (ch >> (lev - 1))
        if lev == 1:
            total += n * (2 + 4)
        else:
            total += n * (4 + 4)
    return total


class Pipeline:
    def __init__(self, w, h, frames, chroma="420", depth=4, intra_filter=6, inter_filter=0,
                 device="cuda"):
        self.lib = _lib.load()
        self.w, self.h, self.frames = w, h, frames
        sx, sy = CHROMA[chroma]
        self.comp_sizes = [(w, h), (w // sx, h // sy), (w // sx, h // sy)]
        self.depth = depth
        self.filters = [intra_filter] + [inter_filter] * (frames - 1)
        self.pics = []      # [frame][comp] int16 (h, w)
        self.coeffs = []    # [frame][comp] int32 (ch, cw)
        for _ in range(frames):
            self.pics.append([torch.zeros((ch_, cw_), dtype=torch.int16, device=device)
                              for (cw_, ch_) in self.comp_sizes])
            self.coeffs.append([torch.zeros(padded_size(cw_, ch_, depth)[::-1], dtype=torch.int32,
                                            device=device) for (cw_, ch_) in self.comp_sizes])
        scratch = 0
        for (cw_, ch_) in self.comp_sizes:
            pw, ph = padded_size(cw_, ch_, depth)
            scratch += self.lib.dgpu_dwt_scratch_bytes(pw, ph, depth)
        self.scratch = torch.empty(scratch * frames, dtype=torch.uint8, device=device)

    # -- data ---------------------------------------------------------------------------------
    def load_frames(self, frames_int16):
        """frames_int16: list of (Y, U, V) int16 tensors (any device)."""
        for f, comps in enumerate(frames_int16):
            for c, t in enumerate(comps):
                self.pics[f][c].copy_(t, non_blocking=True)

    def _items(self):
        items = []
        for f in range(self.frames):
            for c in range(3):
                items.append((self.filters[f], self.depth, self.pics[f][c], self.coeffs[f][c]))
        return items

    def _batch(self, direction, stream):
        items = self._items()
        n = len(items)
        rc = self.lib.dgpu_wavelet_transform_batch(
            direction, n,
            _lib.int_array([it[0] for it in items]),
            _lib.int_array([it[1] for it in items]),
            _lib.ptr_array([it[2].data_ptr() for it in items]),
            _lib.int_array([it[2].shape[1] for it in items]),
            _lib.int_array([it[2].shape[0] for it in items]),
            _lib.int_array([it[2].stride(0) for it in items]),
            _lib.ptr_array([it[3].data_ptr() for it in items]),
            _lib.int_array([it[3].shape[1] for it in items]),
            _lib.int_array([it[3].shape[0] for it in items]),
            _lib.int_array([it[3].stride(0) for it in items]),
            self.scratch.data_ptr(), self.scratch.numel(), stream.cuda_stream)
        _lib.check(rc, "dgpu_wavelet_transform_batch")

    # -- stages ---------------------------------------------------------------------------------
    def stages(self):
        return [("dwt_forward", lambda s: self._batch(FORWARD, s)),
                ("dwt_inverse", lambda s: self._batch(BACKWARD, s))]

    def run_step(self, stream, events=None):
        """Run every stage once on `stream`.  events: optional dict name -> (start, end)
        CUDA events recorded around each stage."""
        for name, fn in self.stages():
            if events is not None:
                events[name][0].record(stream)
            fn(stream)
            if events is not None:
                events[name][1].record(stream)

    def algorithmic_bytes(self):
        """Per stage, bytes moved once per step."""
        fwd = 0
        for (cw_, ch_) in self.comp_sizes:
            pw, ph = padded_size(cw_, ch_, self.depth)
            fwd += dwt_algorithmic_bytes(pw, ph, self.depth, FORWARD)
        fwd *= self.frames
        return {"dwt_forward": fwd, "dwt_inverse": fwd}

    def result_tensors(self):
        """What the host-side coder consumes after a step."""
        return [c for fr in self.coeffs for c in fr]
