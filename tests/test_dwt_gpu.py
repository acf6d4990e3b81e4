"""GPU parity of the wavelet transform against the CPU oracle and the reference's golden
fixtures.  Integer work: every comparison is bit-exact."""
import numpy as np
import pytest
import torch

from test_oracle import ramp

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gpu_forward(d, filt, depth, pic, cw=None, ch=None):
    h, w = pic.shape
    if cw is None:
        cw, ch = d.padded_size(w, h, depth)
    p = dev(pic)
    c = torch.full((ch, cw), -7, dtype=torch.int32, device="cuda")
    d.WaveletTransform(depth, filt).Transform(d.FORWARD, p, c)
    return c.cpu().numpy()


def gpu_backward(d, filt, depth, coeff, w, h):
    c = dev(coeff.astype(np.int32))
    p = torch.full((h, w), 99, dtype=torch.int16, device="cuda")
    d.WaveletTransform(depth, filt).Transform(d.BACKWARD, p, c)
    out = p.cpu().numpy()
    assert np.array_equal(c.cpu().numpy(), coeff), "backward must not modify the coefficients"
    return out


def test_golden_fixtures(gpu, golden):
    g = golden("dwt.npz")
    for key in [k[:-5] for k in g.files if k.endswith("_meta")]:
        filt, depth, w, h, cw, ch = (int(v) for v in g[key + "_meta"])
        np.testing.assert_array_equal(gpu_forward(gpu, filt, depth, g[key + "_pic"], cw, ch),
                                      g[key + "_coeff"], err_msg=key)
        np.testing.assert_array_equal(gpu_backward(gpu, filt, depth, g[key + "_noisy"], w, h),
                                      g[key + "_back"], err_msg=key)


SIZES = [(352, 288, 4), (176, 144, 5), (101, 67, 3), (1920, 1080, 4), (960, 540, 4),
         (720, 576, 5), (1280, 720, 3), (640, 360, 4), (24, 16, 2)]


@pytest.mark.parametrize("filt", range(7))
def test_forward_backward_vs_oracle(gpu, oracle, filt):
    rng = np.random.default_rng(filt)
    for (w, h, depth) in SIZES:
        if (oracle.dwt_min_len(filt) > ((h + (1 << depth) - 1) >> depth << 1)):
            continue
        bd = 10 if w >= 1280 else 8
        pic = rng.integers(-(1 << (bd - 1)), 1 << (bd - 1), size=(h, w)).astype(np.int16)
        c_or = oracle.dwt_forward(filt, depth, pic)
        c_gpu = gpu_forward(gpu, filt, depth, pic)
        np.testing.assert_array_equal(c_gpu, c_or, err_msg=f"fwd {filt} {w}x{h} d{depth}")
        noisy = (c_or + rng.integers(-30, 31, size=c_or.shape)).astype(np.int32)
        np.testing.assert_array_equal(gpu_backward(gpu, filt, depth, noisy, w, h),
                                      oracle.dwt_backward(filt, depth, noisy, w, h),
                                      err_msg=f"bwd {filt} {w}x{h} d{depth}")


@pytest.mark.parametrize("filt", range(8))
def test_invertibility_ramp(gpu, filt):
    """unit_tests/wavelet_utils_test.cpp:84-105 on the GPU."""
    pic = ramp(512, 512)
    c = gpu_forward(gpu, filt, 1, pic)
    np.testing.assert_array_equal(gpu_backward(gpu, filt, 1, c, 512, 512), pic)


def test_batch_mixed_filters_and_depths(gpu, oracle):
    rng = np.random.default_rng(11)
    specs = [(176, 144, 0, 4), (352, 288, 6, 3), (120, 96, 2, 5), (200, 80, 3, 2), (64, 64, 1, 4),
             (90, 60, 4, 1)]
    items, pics = [], []
    for (w, h, filt, depth) in specs:
        pic = rng.integers(-512, 512, size=(h, w)).astype(np.int16)
        cw, ch = gpu.padded_size(w, h, depth)
        items.append((filt, depth, dev(pic), torch.zeros((ch, cw), dtype=torch.int32, device="cuda")))
        pics.append(pic)
    gpu.transform_batch(gpu.FORWARD, items)
    for (w, h, filt, depth), pic, it in zip(specs, pics, items):
        np.testing.assert_array_equal(it[3].cpu().numpy(), oracle.dwt_forward(filt, depth, pic))
    for it in items:
        it[2].zero_()
    gpu.transform_batch(gpu.BACKWARD, items)
    for pic, it in zip(pics, items):
        np.testing.assert_array_equal(it[2].cpu().numpy(), pic)


def test_strided_views_and_caller_scratch(gpu, oracle):
    rng = np.random.default_rng(5)
    w, h, depth, filt = 300, 200, 3, 6
    cw, ch = gpu.padded_size(w, h, depth)
    pic = rng.integers(-128, 128, size=(h, w)).astype(np.int16)
    big = torch.zeros((h, w + 37), dtype=torch.int16, device="cuda")
    big[:, :w] = dev(pic)
    cbig = torch.zeros((ch, cw + 19), dtype=torch.int32, device="cuda")
    wt = gpu.WaveletTransform(depth, filt)
    scratch = torch.zeros(wt.scratch_bytes(cw, ch), dtype=torch.uint8, device="cuda")
    wt.Transform(gpu.FORWARD, big[:, :w], cbig[:, :cw], scratch=scratch)
    np.testing.assert_array_equal(cbig[:, :cw].cpu().numpy(), oracle.dwt_forward(filt, depth, pic))
    assert int(cbig[:, cw:].abs().sum()) == 0


def test_error_codes(gpu):
    wt = gpu.WaveletTransform(4, 0)
    p = torch.zeros((16, 16), dtype=torch.int16, device="cuda")
    c = torch.zeros((16, 16), dtype=torch.int32, device="cuda")
    with pytest.raises(gpu.DgpuError) as e:
        wt.Transform(gpu.FORWARD, p, c)  # level side 2 < 6 for DD9_7
    assert e.value.code == -2
    with pytest.raises(gpu.DgpuError):
        gpu.WaveletTransform(3, 1).Transform(gpu.FORWARD, p, torch.zeros((12, 16), dtype=torch.int32,
                                                                          device="cuda"))
    small = torch.zeros(16, dtype=torch.uint8, device="cuda")
    with pytest.raises(gpu.DgpuError) as e:
        gpu.WaveletTransform(2, 1).Transform(gpu.FORWARD, p, c, scratch=small)
    assert e.value.code == -4


def test_host_buffer_entry_point(gpu, oracle):
    import ctypes

    lib = gpu.load()
    rng = np.random.default_rng(9)
    w, h, depth, filt = 352, 288, 4, 0
    pic = rng.integers(-128, 128, size=(h, w)).astype(np.int16)
    coeff = np.zeros((288, 352), np.int32)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    assert lib.dgpu_wavelet_transform_host(0, filt, depth, P(pic), w, h, w, P(coeff), 352, 288, 352) == 0
    np.testing.assert_array_equal(coeff, oracle.dwt_forward(filt, depth, pic))
    out = np.zeros_like(pic)
    assert lib.dgpu_wavelet_transform_host(1, filt, depth, P(out), w, h, w, P(coeff), 352, 288, 352) == 0
    np.testing.assert_array_equal(out, pic)
