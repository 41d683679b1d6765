"""Pyramid construction and control-point grid refinement (the registration's level set-up)
against the reference CPU library (oracle/_ref):

* nrb_image_pyramid vs reg_createImagePyramid<float> (reg-lib/cpu/_reg_tools.cpp:1705-1733, with
  reg_downsampleImage, :1343-1500): level dims and sform matrices equal (CPU, host-only
  headers); level data with the same NaN pattern and every value within 1e-6 of the level's
  largest magnitude (GPU; the Gaussian smoothing sums in double in both, and the ratio of the
  value and density sums is rounded once);
* nrb_refine_control_point_grid vs reg_spline_refineControlPointGrid3D
  (reg-lib/cpu/_reg_localTrans.cpp:1809-2119) onto the next finer reference: every node value
  within 4 float ulps of the reference's (GPU; sums of up to 27 terms weighted 1 to 216), on even and odd dims and a grid whose spacing is
  not a whole number of voxels. The refined values are the same weighted sums (weights 1, 6, 36,
  216 over 8, 32, 128, 512); the reference writes each of its 24 (case, component) sums with
  its own term order, which this kernel does not reproduce, so the last bit differs on a
  quarter of the nodes.
"""
import numpy as np
import pytest

import niftyreg_b200 as nrb
import oracle
from niftyreg_b200 import phantom
from tests.helpers import ensure_built, identity_grid

PYRAMIDS = {
    # (nz, ny, nx), pixdim (dx, dy, dz), origin, levels
    "even": ((64, 80, 96), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), 3),
    "odd": ((67, 91, 75), (1.0, 1.2, 0.9), (-20.5, 11.0, 3.25), 3),
    "thin_axis": ((40, 130, 129), (0.8, 0.8, 1.5), (5.0, -7.0, 0.0), 3),  # z stops halving
}


def _ref():
    ensure_built()
    if not oracle.ref_available():
        pytest.skip("reference library (oracle/_ref) not built")
    return oracle.Ref()


def _case(name):
    shape, pix, origin, levels = PYRAMIDS[name]
    nz, ny, nx = shape
    img = phantom.blobs_pair(shape, seed=len(name)).reference.astype(np.float32)
    img[0, 0, :3] = np.nan  # NaN voxels travel through the smoothing and the sampling
    xyz = nrb.identity_header(pix, origin)
    return img, (nx, ny, nz), pix, xyz, levels


@pytest.mark.parametrize("name", list(PYRAMIDS))
def test_pyramid_headers_match_reference(name):
    R = _ref()
    img, dim, pix, xyz, levels = _case(name)
    want = R.image_pyramid(img.ravel(), dim, pix, xyz, levels)
    dims, mats, total = nrb.image_pyramid_headers(dim, pix, xyz, levels)
    assert total == sum(int(np.prod(d)) for _, d, _ in want)
    for l, (_, d, m) in enumerate(want):
        assert tuple(dims[l]) == d, (l, dims[l], d)
        assert np.array_equal(mats[l], m), (l, mats[l], m)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(PYRAMIDS))
def test_pyramid_levels_match_reference(name):
    import torch
    R = _ref()
    img, dim, pix, xyz, levels = _case(name)
    want = R.image_pyramid(img.ravel(), dim, pix, xyz, levels)
    _, _, total = nrb.image_pyramid_headers(dim, pix, xyz, levels)
    out = torch.empty(total, dtype=torch.float32, device="cuda")
    nrb.image_pyramid(torch.from_numpy(img.ravel().copy()).cuda(), dim, pix, xyz, levels, out)
    got = out.cpu().numpy()
    off = 0
    for l, (w, d, _) in enumerate(want):
        n = int(np.prod(d))
        g = got[off:off + n]
        off += n
        w = w.ravel()
        assert np.array_equal(np.isnan(g), np.isnan(w)), l
        ok = ~np.isnan(w)
        err = np.abs(g[ok] - w[ok]).max() / np.abs(w[ok]).max()
        print(f"[pyramid] {name} level {l} {d}: max error {err:.2e} of max, "
              f"{np.mean(g[ok] == w[ok]):.4f} of voxels bit-identical")
        assert err <= 1e-6, (l, err)


REFINES = {
    # reference (nz, ny, nx), pixdim, spacing mm at the coarse level
    "even": ((64, 64, 64), (1.0, 1.0, 1.0), 10.0),
    "odd": ((67, 91, 75), (1.0, 1.2, 0.9), 10.0),
    "aniso": ((40, 130, 129), (0.8, 0.8, 1.5), 7.0),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(REFINES))
def test_grid_refinement_matches_reference(name):
    import torch
    R = _ref()
    shape, pix, spacing = REFINES[name]
    nz, ny, nx = shape
    rdim = (nx, ny, nz)
    rxyz = nrb.identity_header(pix, (1.5, -2.0, 0.5))
    # the coarse grid over the reference, displaced, then refined onto the same reference at half
    # the spacing (the registration's refinement onto the next finer level)
    cpp0, cdim, cpix, cxyz = R.create_control_point_grid(rdim, pix, rxyz, (spacing,) * 3)
    rng = np.random.default_rng(len(name))
    cpp = (cpp0 + rng.normal(0, 2.0, cpp0.size)).astype(np.float32)
    want, ndim, npix, nxyz = R.refine_grid(cpp, cdim, cpix, cxyz, rdim, pix, rxyz)
    out = torch.zeros(want.size, dtype=torch.float32, device="cuda")
    nrb.refine_control_point_grid(torch.from_numpy(cpp).cuda(), cdim, out, ndim)
    got = out.cpu().numpy()
    diff = np.abs(got - want)
    # ulps at the scale of the summed node values: a node near the origin is a sum of terms of
    # the order of the grid spacing, whose rounding does not shrink with the result
    ulps = diff / np.spacing(np.maximum(np.abs(want), np.float32(spacing)))
    print(f"[refine] {name}: {tuple(int(v) for v in cdim)} -> {tuple(int(v) for v in ndim)} nodes, "
          f"max |diff| {diff.max():.3g} ({ulps.max():.1f} ulp), {np.mean(got == want):.4f} bit-identical")
    assert ulps.max() <= 4.0
