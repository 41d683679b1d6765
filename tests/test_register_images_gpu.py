"""Registrations of images that carry their own geometry (reg_f3d with -ref / -flo images of any
size, spacing and orientation), through nrb_f3d_register_images and the NIfTI request path
nrb_f3d_register_files.

- an identity-oriented pair gives, bit for bit, the registration of the dims + spacing entry point;
- a reference with a rotated sform and a floating image with other dims, spacings and its own
  rotation: the grid's dims and voxel -> mm matrix are the reference's reg_createControlPointGrid
  ones, and the final NMI agrees with the reference's reg_f3d<float> (oracle/_ref) on the same
  images within the end-point bar of the other registration parity tests (5e-3 relative);
- the file request writes a grid and a warped image that read back as the in-memory results.
"""
import math

import numpy as np
import pytest

import niftyreg_b200 as nrb
from niftyreg_b200 import phantom
from tests.helpers import ensure_built, identity_grid

pytestmark = pytest.mark.gpu


def rotation(ax, ay, az):
    cx, sx, cy, sy, cz, sz = math.cos(ax), math.sin(ax), math.cos(ay), math.sin(ay), math.cos(az), math.sin(az)
    rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return rz @ ry @ rx


def affine(rot, pixdim, origin):
    m = np.eye(4)
    m[:3, :3] = rot @ np.diag(pixdim)
    m[:3, 3] = origin
    return m.astype(np.float32)


class OrientedPair:
    """The blob phantom with the reference placed in the world by a rotated sform, and the
    floating image resampled (trilinear, 0 outside) onto its own grid: other dims, anisotropic
    spacing, another rotation, centred on the reference."""

    def __init__(self, shape=(48, 64, 70), seed=41):
        from scipy import ndimage
        p = phantom.blobs_pair(shape, seed=seed)
        self.ref = p.reference
        nz, ny, nx = shape
        self.rdim, self.rpix = (nx, ny, nz), (1.0, 1.0, 1.0)
        self.rxyz = affine(rotation(0.09, 0.0, 0.21), self.rpix, (-31.0, -27.5, -22.0))
        self.fdim, self.fpix = (66, 60, 56), (0.9, 0.95, 1.1)
        frot = rotation(0.0, -0.14, 0.05)
        centre = self.rxyz.astype(np.float64) @ np.array([(nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2, 1.0])
        fc = np.array([(n - 1) / 2 for n in self.fdim])
        self.fxyz = affine(frot, self.fpix, centre[:3] - frot @ (np.array(self.fpix) * fc))
        k, j, i = np.meshgrid(*[np.arange(n) for n in self.fdim[::-1]], indexing="ij")
        vox = np.stack([i.ravel(), j.ravel(), k.ravel(), np.ones(i.size)])
        u = np.linalg.inv(self.rxyz.astype(np.float64)) @ (self.fxyz.astype(np.float64) @ vox)
        flo = ndimage.map_coordinates(p.floating, [u[2], u[1], u[0]], order=1, mode="constant", cval=0.0)
        self.flo = flo.reshape(self.fdim[::-1]).astype(np.float32)


@pytest.fixture(scope="module")
def oriented():
    ensure_built()
    import torch
    torch.cuda.set_device(0)
    return OrientedPair()


def _params(**kw):
    base = dict(levels=2, max_iterations=40, bending_energy=0.005, spacing=(-5.0,), ref_bins=64, flo_bins=64)
    base.update(kw)
    return nrb.default_params(**base)


def test_identity_images_are_the_dims_and_spacing_registration():
    ensure_built()
    p = phantom.blobs_pair((40, 44, 48), seed=42)
    params = _params()
    cpp, res = nrb.register_host(p.reference, p.floating, p.pixdim, params)
    eye = nrb.identity_header(p.pixdim)
    grid, gxyz, warped, r = nrb.register_images(p.reference, p.pixdim, eye, p.floating, p.pixdim, eye, params)
    assert r.objective_evaluations == res.objective_evaluations
    assert r.final_nmi == res.final_nmi
    assert np.array_equal(grid.ravel(), cpp.ravel())
    nz, ny, nx = p.reference.shape
    _, _, cxyz = nrb.control_grid_header((nx, ny, nz), p.pixdim, [5.0 * v for v in p.pixdim])
    assert np.array_equal(gxyz, cxyz)
    assert warped.shape == p.reference.shape


@pytest.mark.parametrize("padding", [float("nan"), 0.0])
def test_partial_overlap_margins_change_nothing(oriented, padding):
    """A floating image covering a third of the reference's space: most samples fall far outside
    it, beyond any margin, where the texture path clamps its footprints into the margin and the
    dense path selects the padding value per tap; margins 0, 2 and 8, with and without the
    texture, give the same registration bit for bit."""
    o = oriented
    flo = np.ascontiguousarray(o.flo[:, :, :22])
    runs = [nrb.register_images(o.ref, o.rpix, o.rxyz, flo, o.fpix, o.fxyz,
                                _params(floating_margin=m, floating_texture=t, padding=padding), warped=False)
            for m, t in ((0, 0), (2, 1), (8, 1), (8, 0))]
    g0, _, _, r0 = runs[0]
    assert r0.objective_evaluations > 0
    for g, _, _, r in runs[1:]:
        assert r.objective_evaluations == r0.objective_evaluations
        assert r.gradient_evaluations == r0.gradient_evaluations
        assert r.final_nmi == r0.final_nmi
        assert np.array_equal(g, g0)


def test_oriented_images_match_the_reference(oriented):
    import oracle
    if not oracle.ref_available():
        pytest.skip("oracle/_ref/libnrref.so not built")
    o = oriented
    grid, gxyz, warped, r = nrb.register_images(o.ref, o.rpix, o.rxyz, o.flo, o.fpix, o.fxyz, _params())
    R = oracle.Ref()
    R.set_threads(8)
    c_ref, cdim, cxyz_ref, st = R.f3d_register2(o.ref.ravel(), o.rdim, o.rpix, o.rxyz, o.flo.ravel(), o.fdim,
                                                o.fpix, o.fxyz, 2, 40, 0.005, 0.0, 64, -5.0)
    assert list(cdim) == list(r.cpp_dim) == [grid.shape[3], grid.shape[2], grid.shape[1]]
    assert np.allclose(gxyz, cxyz_ref, rtol=0, atol=1e-5), (gxyz, cxyz_ref)
    nmi_ref = st[0]
    print(f"final NMI b200 {r.final_nmi:.8f} reference {nmi_ref:.8f}; evaluations "
          f"{r.objective_evaluations}/{r.gradient_evaluations} vs {int(st[2])}/{int(st[3])}; "
          f"max |cpp diff| {np.abs(c_ref - grid.ravel()).max():.4g} mm")
    assert abs(r.final_nmi - nmi_ref) <= 5e-3 * nmi_ref
    assert r.final_nmi >= (1.0 - 1e-3) * nmi_ref
    # the warped image lives on the reference grid and is closer to it than the floating image
    # resampled with no deformation; the floating field of view (59 mm across x against the
    # reference's 70) leaves about 30 % of the reference padded (NaN)
    assert warped.shape == o.ref.shape
    ok = np.isfinite(warped)
    assert ok.mean() > 0.5
    flo_on_ref = OrientedIdentity(o)
    both = ok & np.isfinite(flo_on_ref)
    err = lambda a: float(np.mean((a[both].astype(np.float64) - o.ref[both]) ** 2))
    assert err(warped) < 0.8 * err(flo_on_ref)


def OrientedIdentity(o):
    """The floating image on the reference grid through the two matrices alone (no deformation):
    a zero-displacement grid warped by the library."""
    import torch
    nz, ny, nx = o.ref.shape
    cdim, cpix, _ = nrb.control_grid_header(o.rdim, o.rpix, [5.0] * 3)
    cxyz = o.rxyz.astype(np.float64).copy()
    cxyz[:3, :3] *= 5.0
    cxyz[:3, 3] = o.rxyz[:3, 3] - cxyz[:3, :3].sum(axis=1)
    cxyz = cxyz.astype(np.float32)
    pos = identity_grid(cdim, cxyz)
    g = nrb.make_geometry(o.rdim, o.rpix, o.rxyz, o.fdim, o.fpix, o.fxyz, cdim, cpix, cxyz)
    w = torch.empty(nx * ny * nz, dtype=torch.float32, device="cuda")
    nrb.f3d_warped_image(g, torch.from_numpy(o.flo.ravel()).cuda(), torch.from_numpy(pos).cuda(), w)
    torch.cuda.synchronize()
    return w.cpu().numpy().reshape(nz, ny, nx)


def test_file_request_reads_back_as_the_image_results(oriented, tmp_path):
    o = oriented
    params = _params(levels=1, max_iterations=15)
    nrb.write_image(tmp_path / "ref.nii.gz", o.ref, o.rpix, o.rxyz)
    nrb.write_image(tmp_path / "flo.nii", o.flo, o.fpix, o.fxyz)
    res = nrb.register_files(tmp_path / "ref.nii.gz", tmp_path / "flo.nii", params, tmp_path / "cpp.nii.gz",
                             tmp_path / "res.nii")
    grid, gxyz, warped, r = nrb.register_images(o.ref, o.rpix, o.rxyz, o.flo, o.fpix, o.fxyz, params)
    assert res.final_nmi == r.final_nmi and res.objective_evaluations == r.objective_evaluations
    c, cpix, cxyz = nrb.read_image(tmp_path / "cpp.nii.gz")
    assert c.shape == grid.shape and np.array_equal(c, grid)
    assert cpix == (5.0, 5.0, 5.0) and np.array_equal(cxyz, gxyz)
    w, wpix, wxyz = nrb.read_image(tmp_path / "res.nii")
    assert np.array_equal(w[0], warped, equal_nan=True)
    assert wpix == o.rpix and np.allclose(wxyz, o.rxyz, atol=1e-6)


def test_refusals(tmp_path):
    ensure_built()
    params = _params(levels=1, max_iterations=2)
    with pytest.raises(nrb.NrbError):
        nrb.register_files(tmp_path / "missing.nii", tmp_path / "missing.nii", params, tmp_path / "cpp.nii")
    a = np.zeros((1, 8, 8), np.float32)  # a 2D image
    eye = np.eye(4, dtype=np.float32)
    with pytest.raises(nrb.NrbError):
        nrb.register_images(a, (1.0, 1.0, 1.0), eye, a, (1.0, 1.0, 1.0), eye, params)
