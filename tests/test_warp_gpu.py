"""The final warp of a registration (reg_f3d::GetWarpedImage, which the reference runs on the CPU
with cubic-spline interpolation) and the order-0/1/3 resampling behind it, through the C ABI.

Tolerance: none. The kernels keep the reference's float operations unfused, so every voxel,
NaN padding included, must be the same float as NiftyReg's own ResampleImage3D (golden fixtures
made by tests/golden/make_golden.py) and as the oracle's restatement.
"""
import glob
import math
import os

import numpy as np
import pytest

import niftyreg_b200 as nrb
import oracle
from niftyreg_b200 import phantom
from tests.helpers import ensure_built, make_case

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.fixture(scope="module")
def O():
    ensure_built()
    return oracle.Restated()


@pytest.fixture(params=CASES, ids=[os.path.basename(c)[:-4] for c in CASES])
def gold(request):
    ensure_built()
    g = dict(np.load(request.param))
    g["geom"] = nrb.make_geometry(tuple(g["rdim"]), tuple(g["rpix"]), g["rxyz"], tuple(g["fdim"]), tuple(g["fpix"]),
                                  g["fxyz"], tuple(g["cdim"]), tuple(g["cpix"]), g["cxyz"])
    return g


def test_orders_match_the_reference_bitwise(gold):
    g = gold
    d, flo = dev(g["def"]), dev(g["flo"])
    for order, key, pad in ((0, "warped_nn", math.nan), (1, "warped", math.nan), (3, "warped_cubic", math.nan),
                            (3, "warped_cubic_pad0", 0.0)):
        w = torch.empty(g[key].size, dtype=torch.float32, device="cuda")
        nrb.resample_image_order(g["geom"], flo, d, w, order, padding=pad)
        assert np.array_equal(host(w), g[key], equal_nan=True), key


def test_orders_match_the_oracle_with_large_displacements(O):
    """Another floating geometry and 4 mm control-point displacements: many windows leave the
    volume, so the padding path runs for many voxels; three padding values."""
    c = make_case(shape=(20, 22, 24), flo_shape=(18, 22, 26), flo_pixdim=(1.2, 1.1, 0.9), seed=33, disp=4.0)
    g = c.geometry()
    dfield = O.deformation_field(c.cpp, c.cdim, c.cpix, c.rdim, c.rpix)
    for order in (0, 1, 3):
        for pad in (math.nan, 0.0, -3.5):
            w = torch.empty(c.nvox, dtype=torch.float32, device="cuda")
            nrb.resample_image_order(g, dev(c.flo), dev(dfield), w, order, padding=pad)
            ref = O.resample_order(c.flo, c.fdim, c.flo_ijk, dfield, c.rdim, order, pad=pad)
            assert np.array_equal(host(w), ref, equal_nan=True), (order, pad)


def test_mask_leaves_voxels_untouched(O):
    c = make_case(seed=34, disp=2.0)
    g = c.geometry()
    rng = np.random.default_rng(34)
    mask = np.where(rng.random(c.nvox) < 0.3, -1, 0).astype(np.int32)
    dfield = O.deformation_field(c.cpp, c.cdim, c.cpix, c.rdim, c.rpix)
    init = np.full(c.nvox, -7.0, np.float32)
    w = dev(init)
    nrb.resample_image_order(g, dev(c.flo), dev(dfield), w, 3, mask=dev(mask))
    ref = O.resample_order(c.flo, c.fdim, c.flo_ijk, dfield, c.rdim, 3, mask=mask, warped_init=init)
    out = host(w)
    assert np.all(out[mask < 0] == -7.0)
    assert np.array_equal(out, ref, equal_nan=True)


def test_warped_image_is_deformation_then_resample():
    c = make_case(shape=(30, 26, 34), seed=35, disp=2.0)
    g = c.geometry()
    flo, cpp = dev(c.flo), dev(c.cpp)
    a = torch.empty(c.nvox, dtype=torch.float32, device="cuda")
    nrb.f3d_warped_image(g, flo, cpp, a)
    d = torch.empty(3 * c.nvox, dtype=torch.float32, device="cuda")
    nrb.get_deformation_field(g, cpp, d)
    b = torch.empty(c.nvox, dtype=torch.float32, device="cuda")
    nrb.resample_image_order(g, flo, d, b, 3)
    assert np.array_equal(host(a), host(b), equal_nan=True)


def test_unsupported_order_is_refused():
    c = make_case(seed=36)
    g = c.geometry()
    w = torch.empty(c.nvox, dtype=torch.float32, device="cuda")
    d = torch.zeros(3 * c.nvox, dtype=torch.float32, device="cuda")
    with pytest.raises(nrb.NrbError):
        nrb.resample_image_order(g, dev(c.flo), d, w, 2)
    with pytest.raises(nrb.NrbError):
        nrb.f3d_warped_image(g, dev(c.flo), dev(c.cpp), w, order=4)


def test_registration_then_warped_image():
    """A whole registration, then its final warp with the registration's grid: the warped image
    is closer to the reference than the floating image is."""
    pair = phantom.blobs_pair((40, 44, 48), seed=37)
    params = nrb.default_params(levels=2, max_iterations=40, bending_energy=0.005, spacing=(-5.0,),
                                ref_bins=64, flo_bins=64)
    cpp, res = nrb.register_host(pair.reference, pair.floating, pair.pixdim, params)
    nz, ny, nx = pair.reference.shape
    dim, pix = (nx, ny, nz), tuple(float(p) for p in pair.pixdim)
    cdim, cpix, cxyz = nrb.control_grid_header(dim, pix, [5.0 * p for p in pix])
    assert list(cdim) == list(res.cpp_dim)
    g = nrb.make_geometry(dim, pix, nrb.identity_header(pix), dim, pix, nrb.identity_header(pix), cdim, cpix, cxyz)
    w = torch.empty(nx * ny * nz, dtype=torch.float32, device="cuda")
    nrb.f3d_warped_image(g, dev(pair.floating.ravel()), dev(cpp.ravel()), w, padding=0.0)
    warped = host(w).reshape(pair.reference.shape)

    def mse(a):
        return float(np.mean((a.astype(np.float64) - pair.reference) ** 2))

    assert mse(warped) < 0.8 * mse(pair.floating)
