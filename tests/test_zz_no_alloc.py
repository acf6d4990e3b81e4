"""The allocation-free wavelet entry point, dgpu_wavelet_transform_static.

It exists for callers that cannot allocate device memory when they transform (a fully
reserved device-memory budget, threads that must not synchronise the device the way
cudaMalloc / cudaFree can, an embedding allocator that owns all device memory): its
intermediates live in one fixed device array instead of caller or library scratch.  These
tests call it through the C ABI and check it against dgpu_wavelet_transform, bit for bit,
on two calls in a row, so that whatever one call leaves in the shared array cannot leak
into the next result.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _run_both(lib, direction, filt, depth, pic_np, coeff_np, stream):
    """Run the same transform through the static and the scratch-taking entry points."""
    h, w = pic_np.shape
    ch, cw = coeff_np.shape
    out = []
    for fn in ("static", "scratch"):
        pic = torch.from_numpy(pic_np.copy()).cuda()
        coeff = torch.from_numpy(coeff_np.copy()).cuda()
        if fn == "static":
            rc = lib.dgpu_wavelet_transform_static(direction, filt, depth, _ptr(pic), w, h, w, _ptr(coeff),
                                                   cw, ch, cw, stream)
        else:
            rc = lib.dgpu_wavelet_transform(direction, filt, depth, _ptr(pic), w, h, w, _ptr(coeff), cw, ch, cw,
                                            None, 0, stream)
        assert rc == 0, (fn, rc)
        torch.cuda.synchronize()
        out.append((pic.cpu().numpy(), coeff.cpu().numpy()))
    return out


def test_static_matches_scratch_entry_point_two_calls_in_a_row(gpu):
    lib = gpu.load()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(2026)
    # two consecutive forward calls with different pictures, sizes and filters, then two
    # inverse calls: each must match the scratch-taking entry point exactly
    cases = [(1920, 1080, 4, gpu.DAUB9_7), (352, 288, 3, gpu.DD9_7)]
    for (w, h, depth, filt) in cases:
        cw, ch = gpu.padded_size(w, h, depth)
        pic = rng.integers(-128, 128, size=(h, w)).astype(np.int16)
        (sp, sc), (rp, rc_) = _run_both(lib, gpu.FORWARD, filt, depth, pic, np.zeros((ch, cw), np.int32), stream)
        np.testing.assert_array_equal(sc, rc_)
    for (w, h, depth, filt) in cases:
        cw, ch = gpu.padded_size(w, h, depth)
        coeff = rng.integers(-600, 600, size=(ch, cw)).astype(np.int32)
        (sp, sc), (rp, rc_) = _run_both(lib, gpu.BACKWARD, filt, depth, np.zeros((h, w), np.int16), coeff, stream)
        np.testing.assert_array_equal(sp, rp)


def test_static_round_trip_and_size_limit(gpu):
    lib = gpu.load()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(7)
    w, h, depth, filt = 960, 540, 4, gpu.LEGALL5_3
    cw, ch = gpu.padded_size(w, h, depth)
    pic_np = rng.integers(-512, 512, size=(h, w)).astype(np.int16)
    pic = torch.from_numpy(pic_np).cuda()
    coeff = torch.zeros((ch, cw), dtype=torch.int32, device="cuda")
    assert lib.dgpu_wavelet_transform_static(0, filt, depth, _ptr(pic), w, h, w, _ptr(coeff), cw, ch, cw,
                                             stream) == 0
    back = torch.zeros_like(pic)
    assert lib.dgpu_wavelet_transform_static(1, filt, depth, _ptr(back), w, h, w, _ptr(coeff), cw, ch, cw,
                                             stream) == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(back.cpu().numpy(), pic_np)
    # a 3840 x 2160 component needs more than the fixed array holds: rejected, nothing launched
    big_w, big_h = 3840, 2160
    assert lib.dgpu_dwt_scratch_bytes(big_w, big_h, 4) > 4 << 20
    rc = lib.dgpu_wavelet_transform_static(0, filt, 4, _ptr(pic), big_w, big_h, big_w, _ptr(coeff), big_w,
                                           big_h, big_w, stream)
    assert rc == -2  # DGPU_ERR_SIZE


_NO_ALLOC_CHILD = r"""
import ctypes, os, sys
sys.path.insert(0, sys.argv[1])
import dirac_b200
lib = dirac_b200.load()          # library registered before the context exists (eager loading)
import torch
w, h, depth = 1920, 1080, 4
cw, ch = dirac_b200.padded_size(w, h, depth)
pic = torch.randint(-128, 128, (h, w), dtype=torch.int16, device="cuda")
coeff = torch.zeros((ch, cw), dtype=torch.int32, device="cuda")
back = torch.zeros_like(pic)
torch.cuda.synchronize()
P = lambda t: ctypes.c_void_p(t.data_ptr())
def static_pair():
    assert lib.dgpu_wavelet_transform_static(0, 6, depth, P(pic), w, h, w, P(coeff), cw, ch, cw, None) == 0
    assert lib.dgpu_wavelet_transform_static(1, 6, depth, P(back), w, h, w, P(coeff), cw, ch, cw, None) == 0
    torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info()[0]
static_pair()                    # the first call on the device (symbol lookup)
free1 = torch.cuda.mem_get_info()[0]
for _ in range(4):
    static_pair()
free2 = torch.cuda.mem_get_info()[0]
assert torch.equal(back, pic)
# the same measurement sees the scratch-taking entry point's library buffer being created
assert lib.dgpu_wavelet_transform(0, 6, depth, P(pic), w, h, w, P(coeff), cw, ch, cw, None, 0, None) == 0
torch.cuda.synchronize()
free3 = torch.cuda.mem_get_info()[0]
print(free0, free1, free2, free3)
"""


def test_static_entry_point_allocates_nothing(gpu):
    """In a fresh process with every module loaded eagerly: device free memory is the same
    before the first static call, after it and after four more forward + inverse pairs; the
    scratch-taking entry point with NULL scratch, run afterwards, does lower it (the library's
    own buffer), so the measurement would see an allocation on the static path."""
    import os
    import subprocess
    import sys

    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "dirac-research_b200")
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    r = subprocess.run([sys.executable, "-c", _NO_ALLOC_CHILD, pkg], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    free0, free1, free2, free3 = map(int, r.stdout.split()[-4:])
    assert free0 == free1 == free2, (free0, free1, free2)
    assert free3 < free2, (free2, free3)
