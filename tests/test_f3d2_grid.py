"""The final grids of F3D and F3D2 registrations from the image headers alone (host only), against
the final grids of the reference's own registrations (oracle/_ref, two iterations per level) on
the CPU:
- nrb_f3d2_grid_header vs reg_f3d2<float>: the symmetric grid over the coarsest pyramid images
  (reg_createSymmetricControlPointGrids), refined once per finer level;
- nrb_f3d_grid_header vs reg_f3d<float>: reg_createControlPointGrid over the coarsest reference,
  refined onto each finer reference.
Dims exact, matrices within 1e-5 mm."""
import numpy as np
import pytest

import niftyreg_b200 as nrb
import oracle
from tests.helpers import ensure_built


@pytest.fixture(scope="module")
def R():
    ensure_built()
    if not oracle.ref_available():
        pytest.skip("oracle/_ref (the reference build) is not present")
    r = oracle.Ref()
    r.set_threads(8)
    return r


def _check(R, rdim, rpix, rxyz, fdim, fpix, fxyz, levels, spacing=-5.0, seed=0):
    rng = np.random.default_rng(seed)
    ref = rng.normal(100, 20, int(np.prod(rdim))).astype(np.float32)
    flo = rng.normal(100, 20, int(np.prod(fdim))).astype(np.float32)
    params = nrb.default_params(levels=levels, max_iterations=2, bending_energy=0.005, spacing=(spacing,))
    dim, pix, xyz = nrb.f3d2_grid_header(rdim, rpix, rxyz, fdim, fpix, fxyz, params)
    _, _, cdim, cxyz, _, _ = R.f3d2_register(ref, rdim, rpix, rxyz, flo, fdim, fpix, fxyz, levels, 2, 0.005, 0.0, 64,
                                             spacing)
    assert dim == list(cdim), (dim, list(cdim))
    assert np.allclose(xyz, cxyz, rtol=0, atol=1e-5), (xyz, cxyz)


def test_axis_aligned_pair_two_levels(R):
    _check(R, (48, 44, 40), (1.0, 1.0, 1.0), nrb.identity_header((1.0, 1.0, 1.0)), (44, 40, 36),
           (1.1, 1.1, 1.2), nrb.identity_header((1.1, 1.1, 1.2), (-1.5, 0.8, -0.6)), 2)


def test_rotated_pair_two_levels(R):
    from tests.test_register_images_gpu import affine, rotation
    rpix, fpix = (1.0, 1.0, 1.0), (0.9, 0.95, 1.1)
    _check(R, (70, 64, 48), rpix, affine(rotation(0.09, 0.0, 0.21), rpix, (-31.0, -27.5, -22.0)), (66, 60, 56),
           fpix, affine(rotation(0.0, -0.14, 0.05), fpix, (-26.7, -20.9, -29.8)), 2)


def test_three_levels_and_mm_spacing(R):
    """Two refinements (the x axes halve twice), a spacing given in mm."""
    _check(R, (130, 70, 40), (0.8, 1.0, 1.5), nrb.identity_header((0.8, 1.0, 1.5), (3.0, -2.0, 1.0)),
           (128, 66, 44), (0.85, 1.05, 1.4), nrb.identity_header((0.85, 1.05, 1.4), (1.0, 0.5, -2.0)), 3,
           spacing=6.0)


def _check_f3d(R, rdim, rpix, rxyz, levels, spacing=-5.0, seed=0):
    rng = np.random.default_rng(seed)
    ref = rng.normal(100, 20, int(np.prod(rdim))).astype(np.float32)
    flo = rng.normal(100, 20, int(np.prod(rdim))).astype(np.float32)
    params = nrb.default_params(levels=levels, max_iterations=2, bending_energy=0.005, spacing=(spacing,))
    dim, pix, xyz = nrb.f3d_grid_header(rdim, rpix, rxyz, params)
    _, cdim, cxyz, _ = R.f3d_register2(ref, rdim, rpix, rxyz, flo, rdim, rpix, rxyz, levels, 2, 0.005, 0.0, 64,
                                       spacing)
    assert dim == list(cdim), (dim, list(cdim))
    assert np.allclose(xyz, cxyz, rtol=0, atol=1e-5), (xyz, cxyz)


def test_f3d_grid_of_a_rotated_reference_two_levels(R):
    """The F3D grid follows the reference's orientation (sform columns scaled), over the
    coarsest reference, then refined onto the finest."""
    from tests.test_register_images_gpu import affine, rotation
    rpix = (1.0, 0.9, 1.2)
    _check_f3d(R, (70, 64, 40), rpix, affine(rotation(0.09, -0.1, 0.21), rpix, (-31.0, -27.5, -22.0)), 2)


def test_f3d_grid_three_levels_mm_spacing(R):
    _check_f3d(R, (130, 70, 40), (0.8, 1.0, 1.5), nrb.identity_header((0.8, 1.0, 1.5), (3.0, -2.0, 1.0)), 3,
               spacing=6.0)
