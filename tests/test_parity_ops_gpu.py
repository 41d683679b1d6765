"""Parity of every C-ABI operation with the CPU oracle (oracle/nrb_oracle.c) on seeded inputs.

Tolerances (stated per test): deformation field within 1e-4 voxel; resampled intensities and
spatial gradients within 1e-4 absolute on [2, 65]-scaled images with identical NaN patterns;
integer joint histograms exact; NMI, entropies and log tables within 1e-10 relative; voxel
and node gradients within 1e-5 of the largest magnitude; bending energy within 1e-6 relative.
"""
import math

import numpy as np
import pytest

import niftyreg_b200 as nrb
import oracle
from tests.helpers import ensure_built, make_case

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

CASES = {
    "iso5": dict(),
    "spacing2": dict(shape=(16, 17, 19), spacing_vox=(2.0, 2.0, 2.0), seed=1),
    "aniso": dict(shape=(18, 30, 26), pixdim=(0.8, 0.8, 1.5), spacing_vox=(12.5, 12.5, 20.0 / 3.0), seed=2),
    "flo_geom": dict(shape=(20, 22, 24), flo_shape=(18, 22, 26), flo_pixdim=(1.2, 1.1, 0.9), seed=3, disp=0.8),
    "nan_ref": dict(seed=4, nan_frac=0.02),
    "bins132": dict(seed=5, bins=132),
}


@pytest.fixture(scope="module")
def O():
    ensure_built()
    return oracle.Restated()


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.fixture(params=list(CASES), scope="module")
def case(request):
    return make_case(**CASES[request.param])


def oracle_pipeline(O, c):
    dfield = O.deformation_field(c.cpp, c.cdim, c.cpix, c.rdim, c.rpix)
    warped = O.resample(c.flo, c.fdim, c.flo_ijk, dfield, c.rdim)
    return dfield, warped


def test_deformation_field(O, case):
    c = case
    g = c.geometry()
    d = torch.empty(3 * c.nvox, dtype=torch.float32, device="cuda")
    nrb.get_deformation_field(g, dev(c.cpp), d)
    ref = O.deformation_field(c.cpp, c.cdim, c.cpix, c.rdim, c.rpix)
    diff = np.abs(host(d) - ref).reshape(3, -1)
    vox = diff / np.asarray(c.rpix, np.float32)[:, None]
    assert vox.max() <= 1e-4, f"max field error {vox.max():.3g} voxel"


def test_deformation_field_mask(O):
    c = make_case(seed=7)
    rng = np.random.default_rng(7)
    mask = np.where(rng.random(c.nvox) < 0.3, -1, 0).astype(np.int32)
    g = c.geometry()
    d = torch.empty(3 * c.nvox, dtype=torch.float32, device="cuda")
    nrb.get_deformation_field(g, dev(c.cpp), d, mask=dev(mask))
    ref = O.deformation_field(c.cpp, c.cdim, c.cpix, c.rdim, c.rpix, mask=mask)
    out = host(d).reshape(3, -1)
    assert np.all(out[:, mask < 0] == 0)
    assert np.abs(out - ref.reshape(3, -1)).max() <= 1e-4


def test_resample_and_gradient(O, case):
    c = case
    g = c.geometry()
    dfield, warped_ref = oracle_pipeline(O, c)
    w = torch.empty(c.nvox, dtype=torch.float32, device="cuda")
    nrb.resample_image(g, dev(c.flo), dev(dfield), w)
    wg = host(w)
    assert np.array_equal(np.isnan(wg), np.isnan(warped_ref)), "NaN padding pattern differs"
    ok = np.isfinite(warped_ref)
    assert np.abs(wg[ok] - warped_ref[ok]).max() <= 1e-4
    gr = torch.empty(3 * c.nvox, dtype=torch.float32, device="cuda")
    nrb.get_image_gradient(g, dev(c.flo), dev(dfield), gr)
    gref = O.image_gradient(c.flo, c.fdim, c.flo_ijk, dfield, c.rdim)
    assert np.abs(host(gr) - gref).max() <= 1e-4


def test_resample_padding_and_mask(O):
    c = make_case(seed=8, disp=4.0)
    rng = np.random.default_rng(8)
    mask = np.where(rng.random(c.nvox) < 0.25, -1, 0).astype(np.int32)
    g = c.geometry()
    dfield, _ = oracle_pipeline(O, c)
    init = np.full(c.nvox, -7.0, np.float32)
    for pad in (0.0, math.nan):
        w = dev(init.copy())
        nrb.resample_image(g, dev(c.flo), dev(dfield), w, padding=pad, mask=dev(mask))
        ref = O.resample(c.flo, c.fdim, c.flo_ijk, dfield, c.rdim, mask=mask, pad=pad, warped_init=init)
        out = host(w)
        assert np.all(out[mask < 0] == -7.0), "masked voxels must be left untouched"
        assert np.array_equal(np.isnan(out), np.isnan(ref))
        ok = np.isfinite(ref)
        assert np.abs(out[ok] - ref[ok]).max() <= 1e-4


def test_intensity_rescale(O):
    rng = np.random.default_rng(11)
    img = (rng.normal(100, 40, 5000)).astype(np.float32)
    img[::97] = np.nan
    t = dev(img)
    nrb.intensity_rescale(t, img.size, 2.0, 65.0)
    ref = O.intensity_rescale(img, 2.0, 65.0)
    out = host(t)
    assert np.array_equal(np.isnan(out), np.isnan(ref))
    ok = np.isfinite(ref)
    assert np.array_equal(out[ok], ref[ok]), "double-precision rescale must be bit-exact"


def test_nmi_value_and_tables(O, case):
    c = case
    g = c.geometry()
    _, warped = oracle_pipeline(O, c)
    nmi = nrb.Nmi(c.bins, c.bins)
    v = nrb.nmi_value(nmi, g, dev(c.ref), dev(warped))
    pro, log, ent = nmi.tables()
    v_ref, pro_ref, log_ref, ent_ref = O.nmi_value(c.ref, warped, c.bins, c.bins)
    assert abs(v - v_ref) <= 1e-10 * abs(v_ref)
    assert np.allclose(ent, ent_ref, rtol=1e-10, atol=0)
    assert np.allclose(pro, pro_ref, rtol=1e-10, atol=1e-18)
    assert np.allclose(log, log_ref, rtol=1e-10, atol=1e-12)


def test_nmi_voxel_gradient(O, case):
    _check_nmi_voxel_gradient(O, case)


def test_nmi_voxel_gradient_large_table(O):
    """180 internal bins: the FP32 copy of the log table (131 KB) does not fit in shared memory,
    so the FP64 window on the global table runs; the same bar."""
    _check_nmi_voxel_gradient(O, make_case(seed=6, bins=180))


def _check_nmi_voxel_gradient(O, c):
    g = c.geometry()
    dfield, warped = oracle_pipeline(O, c)
    wgrad = O.image_gradient(c.flo, c.fdim, c.flo_ijk, dfield, c.rdim)
    nmi = nrb.Nmi(c.bins, c.bins)
    nrb.nmi_value(nmi, g, dev(c.ref), dev(warped))
    vg = torch.zeros(3 * c.nvox, dtype=torch.float32, device="cuda")
    nrb.nmi_voxel_gradient(nmi, g, dev(c.ref), dev(warped), dev(wgrad), vg, weight=0.75)
    _, _, log_ref, ent_ref = O.nmi_value(c.ref, warped, c.bins, c.bins)
    ref = O.nmi_voxel_gradient(c.ref, warped, wgrad, c.bins, c.bins, log_ref, ent_ref, 0.75)
    scale = np.abs(ref).max()
    assert scale > 0
    assert np.abs(host(vg) - ref).max() <= 1e-5 * scale


def test_kernel_convolution_cubic(O):
    rng = np.random.default_rng(12)
    dim, pix = (23, 19, 17), (1.0, 1.2, 0.9)
    img = rng.normal(0, 1, 3 * int(np.prod(dim))).astype(np.float32)
    img[rng.random(img.size) < 0.02] = np.nan
    for axis in range(3):
        t = dev(img)
        nrb.kernel_convolution_cubic(t, 3, dim, pix, 5.0, axis)
        ref = O.kernel_convolution_cubic(img, 3, dim, pix, 5.0, axis)
        out = host(t)
        assert np.array_equal(np.isnan(out), np.isnan(ref))
        ok = np.isfinite(ref)
        assert np.abs(out[ok] - ref[ok]).max() <= 1e-5 * np.abs(ref[ok]).max()


def test_convolve_to_nodes(O, case):
    c = case
    g = c.geometry()
    rng = np.random.default_rng(13)
    vgrad = rng.normal(0, 1e-3, 3 * c.nvox).astype(np.float32)
    ws = nrb.Workspace(g)
    node = torch.full((3 * c.ncp,), 123.0, dtype=torch.float32, device="cuda")
    nrb.convolve_voxel_based_gradient(ws, dev(vgrad), node, 0.995)
    _, ref = O.convolve_to_nodes(vgrad, c.rdim, c.rpix, c.ref_ijk, c.cdim, c.cpix, c.cxyz, c.flo_ijk, 0.995)
    scale = np.abs(ref).max()
    assert np.abs(host(node) - ref).max() <= 1e-5 * scale


def test_convolve_to_nodes_nan_free_path_is_exact():
    """The x pass sums NaN-free rows with a check-free loop and takes the per-tap path (conv_at)
    for rows holding a NaN; both must give the same bits. A NaN at voxel (0, 3, 0) sends the
    first block of rows (z = 0, y = 0..7) down the per-tap path; nodes beyond the kernel radius of
    that voxel along x read those rows' x outputs through the y and z passes, so they must equal
    the NaN-free run bit for bit."""
    c = make_case(shape=(24, 24, 48), seed=31)
    g = c.geometry()
    rng = np.random.default_rng(31)
    vgrad = rng.normal(0, 1e-3, 3 * c.nvox).astype(np.float32)
    ws = nrb.Workspace(g)
    a = torch.empty(3 * c.ncp, dtype=torch.float32, device="cuda")
    b = torch.empty(3 * c.ncp, dtype=torch.float32, device="cuda")
    nrb.convolve_voxel_based_gradient(ws, dev(vgrad), a, 0.995)
    v2 = vgrad.copy()
    v2[3 * 48] = np.nan  # component 0, z = 0, y = 3, x = 0
    nrb.convolve_voxel_based_gradient(ws, dev(v2), b, 0.995)
    cx, cy, cz = c.cdim
    na, nb = host(a).reshape(3, cz, cy, cx), host(b).reshape(3, cz, cy, cx)
    assert not np.array_equal(na[0, :, :, :3], nb[0, :, :, :3])  # the NaN changed the nodes near it
    assert np.array_equal(na[..., 5:], nb[..., 5:])


def test_bending_energy(O, case):
    c = case
    g = c.geometry()
    ws = nrb.Workspace(g)
    be = nrb.approx_bending_energy(ws, dev(c.cpp))
    be_ref = O.be_value(c.cpp, c.cdim)
    assert abs(be - be_ref) <= 1e-6 * abs(be_ref)
    grad0 = np.random.default_rng(14).normal(0, 1, 3 * c.ncp).astype(np.float32)
    gt = dev(grad0)
    nrb.approx_bending_energy_gradient(ws, dev(c.cpp), gt, 0.005)
    ref = O.be_gradient(c.cpp, c.cdim, c.cxyz, 0.005, grad_init=grad0)
    delta, delta_ref = host(gt) - grad0, ref - grad0
    assert np.abs(delta - delta_ref).max() <= 1e-5 * np.abs(delta_ref).max()


def test_bending_energy_identity_is_zero():
    # known answer of reg_test_be.cpp: identity and affine grids have zero bending energy
    c = make_case(seed=15, disp=0.0)
    g = c.geometry()
    ws = nrb.Workspace(g)
    assert abs(nrb.approx_bending_energy(ws, dev(c.cpp))) < 1e-9
    grad = torch.zeros(3 * c.ncp, dtype=torch.float32, device="cuda")
    nrb.approx_bending_energy_gradient(ws, dev(c.cpp), grad, 1.0)
    assert host(grad).max() == 0 and host(grad).min() == 0


def test_optimiser_ops(O):
    rng = np.random.default_rng(16)
    nnode = 3000
    grad = rng.normal(0, 2, 3 * nnode).astype(np.float32)
    ml = nrb.get_maximal_length(dev(grad), nnode)
    assert ml == O.max_length(grad, nnode)
    t = dev(grad)
    nrb.normalise_gradient(t, nnode, ml)
    assert np.array_equal(host(t), O.normalise_gradient(grad, nnode, ml))
    best = rng.normal(0, 50, 3 * nnode).astype(np.float32)
    cur = torch.empty_like(t)
    nrb.update_control_point_position(cur, dev(best), dev(grad), -0.37, 3 * nnode)
    assert np.array_equal(host(cur), O.update_control_points(best, grad, -0.37))


def test_conjugate_gradient(O):
    c = make_case(seed=17)
    ws = nrb.Workspace(c.geometry())
    rng = np.random.default_rng(17)
    n = 3 * c.ncp
    g0 = rng.normal(0, 1, n).astype(np.float32)
    g, a1, a2 = dev(g0), torch.empty(n, device="cuda"), torch.empty(n, device="cuda")
    nrb.conjugate_gradient(ws, g, a1, a2, n, True)
    rg, r1, r2 = O.cg_update(g0, np.zeros(n, np.float32), np.zeros(n, np.float32), True)
    assert np.array_equal(host(a1), r1) and np.array_equal(host(a2), r2)
    g1 = rng.normal(0, 1, n).astype(np.float32)
    g = dev(g1)
    nrb.conjugate_gradient(ws, g, a1, a2, n, False)
    rg, r1, r2 = O.cg_update(g1, r1, r2, False)
    # the dot products are reduced in a different (fixed) order: FP64 rounding only
    assert np.abs(host(g) - rg).max() <= 1e-6 * np.abs(rg).max()
    assert np.array_equal(host(a1), r1)
