"""The oracle (oracle/nrb_oracle.c, a plain-C restatement of the reference's F3D path) pinned
against golden fixtures produced by NiftyReg's own CPU code (tests/golden/make_golden.py runs
oracle/_ref/libnrref.so). CPU only. Each step is fed the reference's own inputs for that step,
so a mismatch points at one function."""
import glob
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


@pytest.fixture(scope="module")
def O():
    return oracle.Restated()


@pytest.fixture(params=CASES, ids=[os.path.basename(c)[:-4] for c in CASES])
def gold(request):
    return dict(np.load(request.param))


def _ijk(m):
    return np.linalg.inv(m.astype(np.float64)).astype(np.float32)


def test_fixtures_present():
    assert len(CASES) >= 3


def test_deformation_field(O, gold):
    g = gold
    d = O.deformation_field(g["cpp"], g["cdim"], g["cpix"], g["rdim"], g["rpix"])
    # the reference's SSE build sums the 64 taps in another order: a few ulp of a mm position
    assert np.abs(d - g["def"]).max() <= 5e-5


def test_resample_and_gradient(O, gold):
    g = gold
    w = O.resample(g["flo"], g["fdim"], _ijk(g["fxyz"]), g["def"], g["rdim"])
    assert np.array_equal(np.isnan(w), np.isnan(g["warped"]))
    ok = ~np.isnan(w)
    assert np.abs(w[ok] - g["warped"][ok]).max() <= 1e-5
    gr = O.image_gradient(g["flo"], g["fdim"], _ijk(g["fxyz"]), g["def"], g["rdim"])
    assert np.abs(gr - g["wgrad"]).max() <= 1e-5


def test_resample_nearest_and_cubic_bit_exact(O, gold):
    """ResampleImage3D with the nearest and cubic-spline kernels (the final warp of
    reg_f3d::GetWarpedImage uses the cubic one): the restatement repeats the reference's float
    operations, so every voxel, NaN padding included, is the same float."""
    g = gold
    ijk = _ijk(g["fxyz"])
    for order, key, pad in ((0, "warped_nn", np.nan), (3, "warped_cubic", np.nan), (3, "warped_cubic_pad0", 0.0)):
        w = O.resample_order(g["flo"], g["fdim"], ijk, g["def"], g["rdim"], order, pad=pad)
        assert np.array_equal(w, g[key], equal_nan=True), key


def test_nmi_tables_bit_exact(O, gold):
    g = gold
    b = int(g["bins"])
    v, pro, logt, ent = O.nmi_value(g["ref"], g["warped"], b, b)
    assert v == g["nmi"]
    assert np.array_equal(pro, g["pro"])
    assert np.array_equal(logt, g["logt"])
    assert np.array_equal(ent, g["ent"])


def test_nmi_voxel_gradient(O, gold):
    g = gold
    b = int(g["bins"])
    vg = O.nmi_voxel_gradient(g["ref"], g["warped"], g["wgrad"], b, b, g["logt"], g["ent"], 1.0)
    scale = np.abs(g["vgrad"]).max()
    assert np.abs(vg - g["vgrad"]).max() <= 1e-6 * scale


def test_kernel_convolution(O, gold):
    g = gold
    for axis, key in enumerate(("conv_x", "conv_y", "conv_z")):
        out = O.kernel_convolution_cubic(g["vgrad"], 3, g["rdim"], g["rpix"], float(g["cpix"][axis]), axis)
        ref = g[key]
        assert np.array_equal(np.isnan(out), np.isnan(ref))
        ok = np.isfinite(ref)
        assert np.abs(out[ok] - ref[ok]).max() <= 1e-6 * np.abs(ref[ok]).max()


def test_convolve_to_nodes(O, gold):
    g = gold
    _, node = O.convolve_to_nodes(g["vgrad"], g["rdim"], g["rpix"], _ijk(g["rxyz"]), g["cdim"], g["cpix"],
                                  g["cxyz"], _ijk(g["fxyz"]), 0.995)
    assert np.linalg.norm(node - g["node"]) <= 1e-6 * np.linalg.norm(g["node"])


def test_bending_energy(O, gold):
    g = gold
    be = O.be_value(g["cpp"], g["cdim"])
    assert abs(be - g["be"]) <= 1e-7 * abs(g["be"])
    grad = O.be_gradient(g["cpp"], g["cdim"], g["cxyz"], 0.005)
    assert np.abs(grad - g["be_grad"]).max() <= 1e-6 * np.abs(g["be_grad"]).max()


# ---- known answers the reference's own unit tests check (reg-test/), restated ---------------

def test_identity_grid_gives_voxel_positions(O):
    """reg_test_getDeformationField.cpp: an identity grid maps every voxel to its own position."""
    from tests.helpers import identity_grid
    import niftyreg_b200 as nrb
    rdim, rpix = (11, 9, 7), (1.0, 1.0, 1.0)
    cdim, cpix, cxyz = nrb.control_grid_header(rdim, rpix, (3.0, 3.0, 3.0))
    d = O.deformation_field(identity_grid(cdim, cxyz), cdim, cpix, rdim, rpix).reshape(3, rdim[2], rdim[1], rdim[0])
    z, y, x = np.meshgrid(np.arange(rdim[2]), np.arange(rdim[1]), np.arange(rdim[0]), indexing="ij")
    for comp, v in zip(d, (x, y, z)):
        assert np.abs(comp - v).max() <= 1e-5


def test_bending_energy_of_affine_grid_is_zero(O):
    """reg_test_be.cpp: identity and affine transformations have no bending energy (up to the
    6-decimal rounding of the reference's second-derivative basis tables)."""
    from tests.helpers import identity_grid
    import niftyreg_b200 as nrb
    cdim, _, cxyz = nrb.control_grid_header((16, 16, 16), (1.0, 1.0, 1.0), (4.0, 4.0, 4.0))
    ident = identity_grid(cdim, cxyz)
    assert abs(O.be_value(ident, cdim)) <= 1e-8
    A = np.array([[1.1, 0.05, 0.0], [0.02, 0.95, 0.03], [0.0, 0.01, 1.05]], np.float32)
    p = ident.reshape(3, -1)
    aff = (A @ p + np.array([[1.5], [-2.0], [0.5]], np.float32)).astype(np.float32).ravel()
    assert abs(O.be_value(aff, cdim)) <= 1e-6


def test_nmi_of_identical_images(O):
    """reg_test_nmi.cpp: NMI = (H_r + H_w) / H_rw; for identical images H_rw = H_r = H_w up to
    the Parzen smoothing, so the value lies in (1, 2]."""
    rng = np.random.default_rng(0)
    img = rng.uniform(2, 65, 4096).astype(np.float32)
    v, _, _, ent = O.nmi_value(img, img, 68, 68)
    assert abs(v - (ent[0] + ent[1]) / ent[2]) <= 1e-12
    assert 1.0 < v <= 2.0
