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
from tests.helpers import ensure_built

MAX_VOXELS = 2097152  # NRB_STATIC_CONV_MAX_VOXELS
MAX_TAPS = 511        # NRB_STATIC_CONV_MAX_TAPS


def _call(fn, img_ptr, nvol, dim, pix, spacing, axis):
    d = nrb._I3(*[int(v) for v in dim])
    p = nrb._F3(*[float(v) for v in pix])
    return fn(ctypes.c_void_p(img_ptr), int(nvol), d, p, ctypes.c_float(spacing), int(axis), None)


def test_static_rejects_oversized_volume():
    """Rejected on the host before any CUDA call: the pointer is never touched."""
    ensure_built()
    L = nrb.lib()
    dim = (129, 128, 128)  # one voxel row above the limit
    assert dim[0] * dim[1] * dim[2] > MAX_VOXELS
    st = _call(L.nrb_kernel_convolution_cubic_static, 16, 1, dim, (1.0, 1.0, 1.0), 5.0, 0)
    assert st == 2  # NRB_ERR_UNSUPPORTED
    assert b"NRB_STATIC_CONV_MAX_VOXELS" in L.nrb_last_error()


def test_static_rejects_wide_kernel():
    ensure_built()
    L = nrb.lib()
    # radius = int(2 * 200 / 1) = 400 -> 801 taps > 511
    st = _call(L.nrb_kernel_convolution_cubic_static, 16, 1, (8, 8, 8), (1.0, 1.0, 1.0), 200.0, 0)
    assert st == 2
    assert b"NRB_STATIC_CONV_MAX_TAPS" in L.nrb_last_error()


def test_static_rejects_bad_arguments():
    ensure_built()
    L = nrb.lib()
    assert _call(L.nrb_kernel_convolution_cubic_static, 0, 1, (8, 8, 8), (1.0, 1.0, 1.0), 5.0, 0) == 1
    assert _call(L.nrb_kernel_convolution_cubic_static, 16, 1, (8, 8, 8), (1.0, 1.0, 1.0), 5.0, 3) == 1
    assert _call(L.nrb_kernel_convolution_cubic_static, 16, 0, (8, 8, 8), (1.0, 1.0, 1.0), 5.0, 0) == 1


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
