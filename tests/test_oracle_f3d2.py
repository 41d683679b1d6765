"""The F3D2 restatement (oracle/nrb_oracle.c: velocity flow and squarings, composition, gradient
exponentiation, symmetrisation) pinned to the reference's own functions (oracle/_ref) on the
CPU. Tolerance: none, every value must be the same float.

The cases are small (a 20x18x16 field, anisotropic spacing, non-zero origin) and cover a grid
that does not reach the whole field, so the sliding extrapolation runs for the flow too.
"""
import numpy as np
import pytest

import oracle
from tests.helpers import ensure_built, identity_grid

import niftyreg_b200 as nrb


@pytest.fixture(scope="module")
def both():
    ensure_built()
    if not oracle.ref_available():
        pytest.skip("oracle/_ref (the reference build) is not present")
    r = oracle.Ref()
    r.set_threads(4)
    return r, oracle.Restated()


def case(seed, fdim=(20, 18, 16), fpix=(1.0, 1.1, 0.9), spacing=4.0, amp=2.0, margin=1):
    rng = np.random.default_rng(seed)
    origin = (-3.0, 2.0, 1.5)
    fxyz = nrb.identity_header(fpix, origin)
    gdim = [int(np.ceil(n * p / spacing + 3)) + margin for n, p in zip(fdim, fpix)]
    gxyz = nrb.identity_header((spacing,) * 3, [o - spacing - 0.5 for o in origin])
    ident = identity_grid(gdim, gxyz)
    vel = (ident + rng.normal(0, amp, ident.size)).astype(np.float32)
    return fdim, fpix, fxyz, gdim, (spacing,) * 3, gxyz, vel


@pytest.mark.parametrize("update,amp,margin", [(False, 2.0, 1), (True, 2.0, 1), (True, 25.0, 1), (False, 2.0, -2)])
def test_velocity_deformation_is_the_reference(both, update, amp, margin):
    R, O = both
    fdim, fpix, fxyz, gdim, gpix, gxyz, vel = case(61, amp=amp, margin=margin)
    ref, rs = R.velocity_def_field(vel, gdim, gpix, gxyz, 6, update, fdim, fpix, fxyz)
    out, os_ = O.velocity_def_field(vel, gdim, gxyz, 6, update, fdim, fxyz)
    assert os_ == rs
    assert np.array_equal(out, ref)


def test_composition_is_the_reference(both):
    R, O = both
    fdim, fpix, fxyz, *_ = case(62)
    rng = np.random.default_rng(62)
    n = int(np.prod(fdim))
    k, j, i = np.meshgrid(*[np.arange(v) for v in fdim[::-1]], indexing="ij")
    vox = np.stack([i.ravel(), j.ravel(), k.ravel(), np.ones(n)])
    ident = (fxyz.astype(np.float64) @ vox)[:3].astype(np.float32).ravel()
    apply = (ident + rng.normal(0, 1.0, ident.size)).astype(np.float32)
    pos = (ident + rng.uniform(-5, 5, ident.size)).astype(np.float32)
    assert np.array_equal(O.def_compose(fdim, fxyz, apply, pos), R.def_compose(fdim, fpix, fxyz, apply, pos))


@pytest.mark.parametrize("steps", [6, 7])
def test_gradient_exponentiation_is_the_reference(both, steps):
    R, O = both
    fdim, fpix, fxyz, gdim, gpix, gxyz, vel = case(63, amp=1.5)
    g = np.random.default_rng(63).normal(0, 1, 3 * int(np.prod(fdim))).astype(np.float32)
    ref = R.exponentiate_gradient(fdim, fpix, fxyz, vel, gdim, gpix, gxyz, steps, g)
    out = O.exponentiate_gradient(fdim, fxyz, vel, gdim, gxyz, steps, g)
    assert np.array_equal(out, ref)


def test_symmetrisation_is_the_reference(both):
    R, O = both
    fdim, fpix, fxyz, gdim, gpix, gxyz, vel = case(64)
    rng = np.random.default_rng(64)
    bxyz = gxyz.copy()
    bxyz[:3, 3] += np.float32(0.75)
    fw = (identity_grid(gdim, gxyz) + rng.normal(0, 2, vel.size)).astype(np.float32)
    bw = (identity_grid(gdim, bxyz) + rng.normal(0, 2, vel.size)).astype(np.float32)
    rf, rb = R.symmetrise(gdim, gpix, gxyz, bxyz, fw, bw)
    of, ob = O.symmetrise(gdim, gxyz, bxyz, fw, bw)
    assert np.array_equal(of, rf) and np.array_equal(ob, rb)


def test_squaring_number_rule(both):
    _, O = both
    assert O.lib.orc_velocity_squaring_steps(ctypes_float(-1.0), ctypes_float(2.0)) == 6
    # 0.28 * 2^7 = 35.84: an extremum of 36 mm needs 8 squarings
    assert O.lib.orc_velocity_squaring_steps(ctypes_float(-36.0), ctypes_float(1.0)) == 8


def ctypes_float(v):
    import ctypes
    return ctypes.c_float(v)


def test_restatement_matches_the_committed_reference_outputs():
    """Against the reference's own outputs committed in tests/golden/f3d2/velocity.npz (made by
    make_f3d2_golden.py from oracle/_ref): needs no reference build. Bitwise."""
    import os
    ensure_built()
    O = oracle.Restated()
    g = dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "f3d2", "velocity.npz")))
    fdim, fxyz, gdim, gxyz, vel = tuple(g["fdim"]), g["fxyz"], tuple(g["gdim"]), g["gxyz"], g["vel"]
    d6, s6 = O.velocity_def_field(vel, gdim, gxyz, 6, False, fdim, fxyz)
    assert s6 == 6 and np.array_equal(d6, g["def6"])
    du, su = O.velocity_def_field(vel, gdim, gxyz, 6, True, fdim, fxyz)
    assert su == int(g["steps_upd"]) and np.array_equal(du, g["def_upd"])
    dt, _ = O.velocity_def_field(g["vel_tight"], tuple(g["gdim_tight"]), g["gxyz_tight"], 6, False, fdim, fxyz)
    assert np.array_equal(dt, g["def_tight"])
    assert np.array_equal(O.def_compose(fdim, fxyz, g["apply"], g["pos"]), g["composed"])
    assert np.array_equal(O.exponentiate_gradient(fdim, fxyz, vel, gdim, gxyz, 7, g["vgrad"]), g["expgrad7"])
    sf, sb = O.symmetrise(gdim, gxyz, g["bxyz"], g["fw"], g["bw"])
    assert np.array_equal(sf, g["sym_fw"]) and np.array_equal(sb, g["sym_bw"])


def test_voxel_to_node_for_an_unaligned_grid_is_the_reference(both):
    """Compute::ConvolveVoxelBasedMeasureGradient with a rotated reference under an axis-aligned
    grid (the F3D2 situation): the restatement convolves the whole gradient along the image axes
    and samples every node through the full node -> voxel matrix. Within 1e-6 of the largest
    node value: the convolution sums run in another order than the reference's (as for an
    aligned grid, tests/test_oracle_golden.py); the measured gap is 1.6e-7 relative."""
    from tests.test_register_images_gpu import affine, rotation
    R, O = both
    rdim, rpix = (26, 22, 18), (1.0, 1.1, 0.9)
    rxyz = affine(rotation(0.09, -0.05, 0.21), rpix, (-14.0, -12.5, -9.0))
    fdim, fpix = (24, 20, 20), (1.1, 1.0, 1.0)
    fxyz = affine(rotation(0.0, 0.1, -0.07), fpix, (-12.0, -11.0, -10.0))
    cdim, cpix = (10, 9, 8), (5.0, 5.0, 5.0)
    cxyz = nrb.identity_header(cpix, (-20.0, -18.0, -16.0))
    vg = np.random.default_rng(3).normal(size=3 * int(np.prod(rdim))).astype(np.float32)
    _, ref = R.convolve_to_nodes(vg, rdim, rpix, rxyz, fdim, fpix, fxyz, cdim, cpix, cxyz, 0.7)
    ijk = np.linalg.inv(rxyz.astype(np.float64)).astype(np.float32)
    fijk = np.linalg.inv(fxyz.astype(np.float64)).astype(np.float32)
    _, out = O.convolve_to_nodes(vg, rdim, rpix, ijk, cdim, cpix, cxyz, fijk, 0.7)
    assert float(np.abs(out - ref).max()) <= 1e-6 * float(np.abs(ref).max())


def test_rotated_field(both):
    """A field under a rotated voxel -> mm matrix (an F3D2 image of any orientation) and an
    axis-aligned velocity grid: the flow and squarings stay bitwise (per-voxel basis, no axis
    table). The gradient exponentiation's reorientation is the inverse orthogonal factor of the
    field's matrix; the restatement (as the CUDA path) takes it from a scaled Newton iteration
    in double where niftilib's nifti_mat33_polar iterates in float, so the transported gradient
    agrees within 1e-6 of its largest component (measured 3e-7)."""
    from tests.test_register_images_gpu import affine, rotation
    R, O = both
    fdim, fpix = (20, 18, 16), (1.0, 1.1, 0.9)
    fxyz = affine(rotation(0.12, -0.07, 0.2), fpix, (-9.0, -8.0, -7.0))
    gdim, gpix = (12, 12, 11), (4.0, 4.0, 4.0)
    gxyz = nrb.identity_header(gpix, (-25.0, -24.0, -22.0))
    rng = np.random.default_rng(5)
    vel = (identity_grid(gdim, gxyz) + rng.normal(0, 1.5, 3 * int(np.prod(gdim)))).astype(np.float32)
    ref, rs = R.velocity_def_field(vel, gdim, gpix, gxyz, 6, True, fdim, fpix, fxyz)
    out, os_ = O.velocity_def_field(vel, gdim, gxyz, 6, True, fdim, fxyz)
    assert os_ == rs and np.array_equal(out, ref)
    vg = rng.normal(0, 1, 3 * int(np.prod(fdim))).astype(np.float32)
    ref = R.exponentiate_gradient(fdim, fpix, fxyz, vel, gdim, gpix, gxyz, 6, vg)
    out = O.exponentiate_gradient(fdim, fxyz, vel, gdim, gxyz, 6, vg)
    assert float(np.abs(out - ref).max()) <= 1e-6 * float(np.abs(ref).max())
