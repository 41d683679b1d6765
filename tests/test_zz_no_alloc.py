"""nrb_kernel_convolution_cubic_static: the allocation-free variant of the one-axis cubic
B-spline convolution. Its scratch is a fixed per-device array, so these tests check that it
gives the same volumes as nrb_kernel_convolution_cubic on consecutive calls (stale scratch from
an earlier, larger call must not leak into a later one) and that it refuses what does not fit.

The file name sorts last so that the GPU test also runs after the rest of the suite has used
the device; it passes on its own in a fresh process too.
"""
import ctypes

import numpy as np
import pytest

import niftyreg_b200 as nrb
from tests.helpers import ArgBuffers, ensure_built

MAX_VOXELS = 2097152  # NRB_STATIC_CONV_MAX_VOXELS
MAX_TAPS = 511        # NRB_STATIC_CONV_MAX_TAPS


def _call(fn, img_ptr, nvol, dim, pix, spacing, axis):
    d = nrb._I3(*[int(v) for v in dim])
    p = nrb._F3(*[float(v) for v in pix])
    return fn(ctypes.c_void_p(img_ptr), int(nvol), d, p, ctypes.c_float(spacing), int(axis), None)


def _buf():
    return ArgBuffers(1)


def test_static_rejects_oversized_volume():
    """Rejected on the host before any CUDA call."""
    ensure_built()
    L = nrb.lib()
    b = _buf()
    dim = (129, 128, 128)  # one voxel row above the limit
    assert dim[0] * dim[1] * dim[2] > MAX_VOXELS
    st = _call(L.nrb_kernel_convolution_cubic_static, b[0].value, 1, dim, (1.0, 1.0, 1.0), 5.0, 0)
    assert st == 2  # NRB_ERR_UNSUPPORTED
    assert b"NRB_STATIC_CONV_MAX_VOXELS" in L.nrb_last_error()


def test_static_rejects_wide_kernel():
    ensure_built()
    L = nrb.lib()
    b = _buf()
    # radius = int(2 * 200 / 1) = 400 -> 801 taps > 511
    st = _call(L.nrb_kernel_convolution_cubic_static, b[0].value, 1, (8, 8, 8), (1.0, 1.0, 1.0), 200.0, 0)
    assert st == 2
    assert b"NRB_STATIC_CONV_MAX_TAPS" in L.nrb_last_error()


def test_static_rejects_bad_arguments():
    ensure_built()
    L = nrb.lib()
    b = _buf()
    p = b[0].value
    assert _call(L.nrb_kernel_convolution_cubic_static, 0, 1, (8, 8, 8), (1.0, 1.0, 1.0), 5.0, 0) == 1
    assert _call(L.nrb_kernel_convolution_cubic_static, p, 1, (8, 8, 8), (1.0, 1.0, 1.0), 5.0, 3) == 1
    assert _call(L.nrb_kernel_convolution_cubic_static, p, 0, (8, 8, 8), (1.0, 1.0, 1.0), 5.0, 0) == 1


@pytest.mark.parametrize("fn", ["nrb_kernel_convolution_cubic", "nrb_kernel_convolution_cubic_static"])
def test_voxel_sizes_and_spacings_that_leave_the_kernel_undefined_are_refused(fn):
    """A spacing in mm over a voxel size that is 0, negative, NaN or infinite, or a NaN spacing,
    has no kernel: both entry points refuse it before any device work."""
    ensure_built()
    L = nrb.lib()
    f = getattr(L, fn)
    b = _buf()
    p = b[0].value
    nan, inf = float("nan"), float("inf")
    for pix, spacing in [((0.0, 1.0, 1.0), 5.0), ((-1.0, 1.0, 1.0), 5.0), ((nan, 1.0, 1.0), 5.0),
                         ((inf, 1.0, 1.0), 5.0), ((1.0, 1.0, 1.0), nan), ((1.0, 1.0, 1.0), inf)]:
        assert _call(f, p, 1, (8, 8, 8), pix, spacing, 0) == 1, (pix, spacing)
        assert b"spacing" in L.nrb_last_error()
    # a kernel radius above 2^20 voxels is refused, not truncated
    assert _call(f, p, 1, (8, 8, 8), (1e-6, 1.0, 1.0), 5.0, 0) == 2


def test_flat_axis_is_left_as_is_by_both_entry_points():
    """An axis of one voxel leaves the image unchanged (the reference's early return) whatever
    the kernel width: the allocation-free entry point returns OK like the allocating one, before
    its limit on the number of taps, and neither touches the buffer."""
    ensure_built()
    L = nrb.lib()
    b = _buf()
    p = b[0].value
    for fn in ("nrb_kernel_convolution_cubic", "nrb_kernel_convolution_cubic_static"):
        # 801 taps on the flat x axis: above the static limit, but nothing to convolve
        assert _call(getattr(L, fn), p, 1, (1, 8, 8), (1.0, 1.0, 1.0), 200.0, 0) == 0, fn
        assert _call(getattr(L, fn), p, 1, (8, 8, 8), (1.0, 1.0, 1.0), 0.0, 1) == 0, fn


@pytest.mark.gpu
def test_static_matches_allocating_entry_point():
    import torch

    ensure_built()
    L = nrb.lib()
    torch.cuda.set_device(0)
    rng = np.random.default_rng(21)
    # first a large volume close to the limit, then a small one: the second call must not see
    # anything the first one left in the scratch
    cases = [((160, 128, 100), (1.0, 1.0, 1.2), 5.0, 3), ((23, 19, 17), (1.0, 1.2, 0.9), -2.5, 3)]
    for dim, pix, spacing, nvol in cases:
        nv = int(np.prod(dim))
        assert nv <= MAX_VOXELS
        img = rng.normal(0, 1, nvol * nv).astype(np.float32)
        img[rng.random(img.size) < 0.02] = np.nan
        for axis in range(3):
            a = torch.from_numpy(img).cuda()
            b = torch.from_numpy(img).cuda()
            nrb.check(_call(L.nrb_kernel_convolution_cubic, a.data_ptr(), nvol, dim, pix, spacing, axis))
            # two calls in a row through the static scratch, each checked
            for _ in range(2):
                c = b.clone()
                nrb.check(_call(L.nrb_kernel_convolution_cubic_static, c.data_ptr(), nvol, dim, pix, spacing, axis))
                torch.cuda.synchronize()
                want, got = a.cpu().numpy(), c.cpu().numpy()
                assert np.array_equal(np.isnan(want), np.isnan(got))
                ok = np.isfinite(want)
                # same kernels on the same inputs: the tolerance is there only to state the bar
                assert np.abs(got[ok] - want[ok]).max() <= 1e-6 * np.abs(want[ok]).max()
