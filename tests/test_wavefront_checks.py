"""Failure detection and decision-order audit of the motion-estimation wavefronts.

The reference decides blocks one at a time in raster order; the device decides a block as soon
as the neighbours its predictor reads are final, each wait on a neighbour's completion flag
bounded.  Failure detection: dgpu_debug_wavefront leaves one unit's flag unset, so the waits of
its dependants run out after a short limit; the call must return DGPU_ERR_CUDA with the device
context intact, and the next normal call must succeed with the oracle's results.  No fault,
trap or hang is involved: every wait ends by its own limit.  Order audit: the first task's
wavefronts record the position at which each unit was decided, and every unit must come after
the neighbours its predictor depends on (pel search: left, top, top-right,
pixel_match.cpp:242-349; sub-pel: left, top-left, top, top-right, me_subpel.cpp:120-176; mode
decision: left, top, top-left superblocks, me_mode_decn.cpp)."""
import numpy as np
import pytest

PEL_DEPS = ((-1, 0), (0, -1), (1, -1))
SUBPEL_DEPS = ((-1, 0), (-1, -1), (0, -1), (1, -1))
MODE_DEPS = ((-1, 0), (0, -1), (-1, -1))


def order_violations(order, deps):
    """Units (x, y) of a row-major decision-order grid decided before an in-bounds dependency,
    plus a note if the order is not a permutation (a unit decided twice or never)."""
    h, w = order.shape
    bad = []
    if not np.array_equal(np.sort(order.ravel()), np.arange(order.size)):
        bad.append("not a permutation")
    for y in range(h):
        for x in range(w):
            for dx, dy in deps:
                xx, yy = x + dx, y + dy
                if 0 <= xx < w and 0 <= yy < h and order[yy, xx] >= order[y, x]:
                    bad.append((x, y, xx, yy))
    return bad


def test_order_checker_finds_a_planted_inversion():
    """The checker on the CPU: raster order and an anti-diagonal wavefront order pass; the same
    orders with one dependency inverted, or a unit repeated, fail."""
    h, w = 5, 7
    raster = np.arange(h * w).reshape(h, w)
    assert order_violations(raster, PEL_DEPS) == []
    assert order_violations(raster, SUBPEL_DEPS) == []
    # slope-2 diagonals: t = x + 2y orders left and top-right neighbours first
    keys = sorted(((x + 2 * y, y, x) for y in range(h) for x in range(w)))
    wave = np.zeros((h, w), np.int64)
    for k, (_, y, x) in enumerate(keys):
        wave[y, x] = k
    assert order_violations(wave, PEL_DEPS) == []
    swapped = wave.copy()
    swapped[2, 3], swapped[1, 4] = wave[1, 4], wave[2, 3]  # (4, 1) is (3, 2)'s top-right neighbour
    assert (3, 2, 4, 1) in order_violations(swapped, PEL_DEPS)
    dup = raster.copy()
    dup[3, 3] = dup[3, 2]
    assert "not a permutation" in order_violations(dup, PEL_DEPS)


def _frames():
    from dirac_b200 import synth

    seq = synth.make_sequence(352, 288, 3, n_rects=8, vmax=8, seed=4242)
    return [[synth.to_signed(p) for p in fr] for fr in seq]


def _bp():
    from oracle import BlockParams

    return BlockParams(2, 12, 12, 8, 8, 11, 9)


def _estimate(gpu, f, stages):
    import torch

    bp = _bp()
    bpg = gpu.BlockParams(bp.precision, bp.xblen, bp.yblen, bp.xbsep, bp.ybsep, bp.xnum_sb, bp.ynum_sb)
    dev = [[torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in fr] for fr in f]
    out = gpu.MotionEstimator(bpg, 2).Estimate(dev[1], dev[0], dev[2], 10.0, stages)
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.gpu
@pytest.mark.parametrize("stages", [1, 3])
def test_wait_that_runs_out_returns_an_error_and_the_device_recovers(gpu, oracle, stages):
    import torch

    from dirac_b200._lib import DgpuError

    lib = gpu.load()
    f = _frames()
    try:
        assert lib.dgpu_debug_wavefront(0, 4096, None, None, None, None) == 0
        with pytest.raises(DgpuError) as e:
            _estimate(gpu, f, stages)
        assert e.value.code == -3  # DGPU_ERR_CUDA
    finally:
        assert lib.dgpu_debug_wavefront(-1, 0, None, None, None, None) == 0
    torch.cuda.synchronize()  # the context is usable
    got = _estimate(gpu, f, 3)
    want = oracle.motion_estimate(2, f[1], f[0], f[2], _bp(), 10.0, 3)
    for k, v in want.items():
        np.testing.assert_array_equal(got[k], v, err_msg=k)


@pytest.mark.gpu
def test_wavefront_decision_order_respects_raster_dependencies(gpu, oracle):
    import torch

    lib = gpu.load()
    f = _frames()
    bp = _bp()
    ynb, xnb = 4 * bp.ynum_sb, 4 * bp.xnum_sb
    audits = [torch.zeros(1 + n, dtype=torch.int32, device="cuda")
              for n in (xnb * ynb, xnb * ynb, bp.xnum_sb * bp.ynum_sb)]
    try:
        assert lib.dgpu_debug_wavefront(-1, 0, *[a.data_ptr() for a in audits], None) == 0
        got = _estimate(gpu, f, 3)
    finally:
        assert lib.dgpu_debug_wavefront(-1, 0, None, None, None, None) == 0
    want = oracle.motion_estimate(2, f[1], f[0], f[2], bp, 10.0, 3)
    for k, v in want.items():
        np.testing.assert_array_equal(got[k], v, err_msg=k)
    a = [x.cpu().numpy() for x in audits]
    # the first job of each launch (first task, first reference) records every unit once
    assert a[0][0] == xnb * ynb and a[1][0] == xnb * ynb and a[2][0] == bp.xnum_sb * bp.ynum_sb
    for name, arr, shape, deps in (("pel", a[0], (ynb, xnb), PEL_DEPS), ("subpel", a[1], (ynb, xnb), SUBPEL_DEPS),
                                   ("mode", a[2], (bp.ynum_sb, bp.xnum_sb), MODE_DEPS)):
        assert order_violations(arr[1:].reshape(shape), deps) == [], name


@pytest.mark.gpu
def test_estimates_do_not_depend_on_wavefront_occupancy(gpu, oracle):
    """dgpu_me_set_occupancy changes only how many CTAs of a wavefront launch stay resident per
    SM (down to one, where most units wait for tickets held by other SMs' CTAs): the results
    equal the oracle's at every setting."""
    lib = gpu.load()
    f = _frames()
    want = oracle.motion_estimate(2, f[1], f[0], f[2], _bp(), 10.0, 3)
    try:
        for occ in (1, 3, 8):
            assert lib.dgpu_me_set_occupancy(occ) == 0
            got = _estimate(gpu, f, 3)
            for k, v in want.items():
                np.testing.assert_array_equal(got[k], v, err_msg=f"{k} at {occ} CTAs per SM")
    finally:
        assert lib.dgpu_me_set_occupancy(8) == 0


@pytest.mark.gpu
def test_estimates_do_not_depend_on_unit_lifetime(gpu, oracle):
    """dgpu_me_set_unit_lifetime bounds how many units a warp (a CTA of the mode wavefront)
    takes before it exits, the grid growing to cover the rest: down to one unit per warp, and
    with one resident CTA per SM, the results equal the oracle's."""
    lib = gpu.load()
    f = _frames()
    want = oracle.motion_estimate(2, f[1], f[0], f[2], _bp(), 10.0, 3)
    try:
        for life, occ in ((1, 8), (3, 8), (64, 8), (2, 1)):
            assert lib.dgpu_me_set_unit_lifetime(life) == 0
            assert lib.dgpu_me_set_occupancy(occ) == 0
            got = _estimate(gpu, f, 3)
            for k, v in want.items():
                np.testing.assert_array_equal(got[k], v, err_msg=f"{k} at lifetime {life}, {occ} CTAs per SM")
    finally:
        assert lib.dgpu_me_set_unit_lifetime(0) == 0
        assert lib.dgpu_me_set_occupancy(8) == 0


def test_unit_lifetime_rejects_negative_values():
    from dirac_b200 import _lib

    lib = _lib.load()
    assert lib.dgpu_me_set_unit_lifetime(-1) == -1
    assert lib.dgpu_me_set_unit_lifetime(0) == 0


def test_blocking_waits_switch():
    from dirac_b200 import _lib

    lib = _lib.load()
    assert lib.dgpu_set_blocking_waits(3) == -1 and lib.dgpu_set_blocking_waits(-1) == -1
    for mode in (1, 2, 0):
        assert lib.dgpu_set_blocking_waits(mode) == 0


def test_wavefront_occupancy_rejects_out_of_range_values():
    from dirac_b200 import _lib

    lib = _lib.load()
    assert lib.dgpu_me_set_occupancy(0) == -1 and lib.dgpu_me_set_occupancy(9) == -1
    assert lib.dgpu_me_set_occupancy(8) == 0
