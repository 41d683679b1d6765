"""F3D2 (reg_f3d2, the -vel / -sym registration) through the C ABI, against the reference's own
functions (oracle/_ref) on the same inputs.

Tolerances:
- velocity -> deformation (flow, scaling, N squarings), composition, exponentiated gradient and
  symmetrisation: none. The kernels perform the reference's float operations in its order, unfused
  (its SSE build has no fused multiply-add), so every value is the same float;
- whole registration: the end-point bar of the other registration parity tests (final NMI
  within 5e-3 relative, not worse by more than 1e-3), grids of the same dims and matrix. The NMI
  histograms and the bending energy are summed in another order, so the trajectories part after
  a few line-search decisions.
"""
import numpy as np
import pytest

import niftyreg_b200 as nrb
import oracle
from niftyreg_b200 import phantom
from tests.helpers import ensure_built, identity_grid

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.fixture(scope="module")
def R():
    ensure_built()
    if not oracle.ref_available():
        pytest.skip("oracle/_ref (the reference build) is not present")
    r = oracle.Ref()
    r.set_threads(8)
    return r


class VelocityCase:
    """An axis-aligned field (anisotropic spacing, non-zero origin) and a velocity grid over it
    with one node of margin: identity positions plus smooth random node displacements."""

    def __init__(self, seed, fdim=(30, 26, 22), fpix=(1.0, 1.1, 0.9), spacing=5.0, amp=2.5):
        rng = np.random.default_rng(seed)
        self.fdim, self.fpix = fdim, fpix
        origin = (-3.0, 2.0, 1.5)
        self.fxyz = nrb.identity_header(fpix, origin)
        self.gdim = [int(np.ceil(n * p / spacing + 3)) + 1 for n, p in zip(fdim, fpix)]
        self.gpix = (spacing,) * 3
        self.gxyz = nrb.identity_header(self.gpix, [o - spacing - 0.5 for o in origin])
        ident = identity_grid(self.gdim, self.gxyz)
        self.vel = (ident + rng.normal(0, amp, ident.size)).astype(np.float32)
        self.n = int(np.prod(fdim))

    def geometry(self):
        return nrb.make_geometry(self.fdim, self.fpix, self.fxyz, self.fdim, self.fpix, self.fxyz, self.gdim,
                                 self.gpix, self.gxyz)


@pytest.mark.parametrize("update", [False, True])
def test_velocity_deformation_matches_reference(R, update):
    c = VelocityCase(51)
    steps_in = 6
    ref_def, ref_steps = R.velocity_def_field(c.vel, c.gdim, c.gpix, c.gxyz, steps_in, update, c.fdim, c.fpix, c.fxyz)
    d = torch.empty(3 * c.n, dtype=torch.float32, device="cuda")
    steps = nrb.get_def_field_from_velocity_grid(c.geometry(), dev(c.vel), steps_in, d, update=update)
    out = host(d)
    err = float(np.abs(out - ref_def).max())
    print(f"steps {steps} (reference {ref_steps}); max |def - reference| {err:.3g} mm")
    assert steps == ref_steps
    assert np.array_equal(out, ref_def)


def test_large_velocity_raises_the_squaring_number(R):
    c = VelocityCase(52, amp=30.0)  # N = 8
    ref_def, ref_steps = R.velocity_def_field(c.vel, c.gdim, c.gpix, c.gxyz, 6, True, c.fdim, c.fpix, c.fxyz)
    d = torch.empty(3 * c.n, dtype=torch.float32, device="cuda")
    steps = nrb.get_def_field_from_velocity_grid(c.geometry(), dev(c.vel), 6, d, update=True)
    assert steps == ref_steps > 6
    assert np.array_equal(host(d), ref_def)


def test_composition_matches_reference(R):
    """Positions reaching up to 6 mm outside the field: the sliding extrapolation runs."""
    c = VelocityCase(53)
    rng = np.random.default_rng(53)
    pos = np.concatenate([np.zeros(c.n, np.float32)] * 3)
    k, j, i = np.meshgrid(*[np.arange(n) for n in c.fdim[::-1]], indexing="ij")
    vox = np.stack([i.ravel(), j.ravel(), k.ravel(), np.ones(c.n)])
    ident = (c.fxyz.astype(np.float64) @ vox)[:3].astype(np.float32).ravel()
    apply = (ident + rng.normal(0, 1.0, ident.size)).astype(np.float32)
    pos = (ident + rng.uniform(-6, 6, ident.size)).astype(np.float32)
    ref = R.def_compose(c.fdim, c.fpix, c.fxyz, apply, pos)
    u = dev(pos)
    nrb.def_field_compose(c.fdim, c.fxyz, dev(apply), u)
    err = float(np.abs(host(u) - ref).max())
    print(f"max |compose - reference| {err:.3g} mm")
    assert np.array_equal(host(u), ref)


def test_exponentiated_gradient_matches_reference(R):
    c = VelocityCase(54, amp=1.5)
    rng = np.random.default_rng(54)
    vgrad = rng.normal(0, 1.0, 3 * c.n).astype(np.float32)
    ref = R.exponentiate_gradient(c.fdim, c.fpix, c.fxyz, c.vel, c.gdim, c.gpix, c.gxyz, 6, vgrad)
    g = dev(vgrad)
    nrb.exponentiate_gradient(c.geometry(), dev(c.vel), 6, g)
    out = host(g)
    err = float(np.abs(out - ref).max())
    print(f"max |exp gradient - reference| {err:.3g} (largest component {np.abs(ref).max():.3g})")
    assert np.array_equal(out, ref)


def test_symmetrisation_is_bitwise(R):
    c = VelocityCase(55)
    rng = np.random.default_rng(55)
    bxyz = c.gxyz.copy()
    bxyz[:3, 3] += np.float32(0.75)
    fw = (identity_grid(c.gdim, c.gxyz) + rng.normal(0, 2, c.vel.size)).astype(np.float32)
    bw = (identity_grid(c.gdim, bxyz) + rng.normal(0, 2, c.vel.size)).astype(np.float32)
    rf, rb = R.symmetrise(c.gdim, c.gpix, c.gxyz, bxyz, fw, bw)
    g_fw = nrb.make_geometry(c.fdim, c.fpix, c.fxyz, c.fdim, c.fpix, c.fxyz, c.gdim, c.gpix, c.gxyz)
    g_bw = nrb.make_geometry(c.fdim, c.fpix, c.fxyz, c.fdim, c.fpix, c.fxyz, c.gdim, c.gpix, bxyz)
    a, b = dev(fw), dev(bw)
    nrb.symmetrise_velocity_fields(g_fw, a, g_bw, b)
    assert np.array_equal(host(a), rf)
    assert np.array_equal(host(b), rb)


def _pair():
    """The blob phantom as the reference (1 mm, origin 0) and its floating image resampled onto
    an axis-aligned grid of other dims and spacing, shifted origin."""
    from scipy import ndimage
    p = phantom.blobs_pair((40, 44, 48), seed=56)
    fdim, fpix = (44, 40, 36), (1.1, 1.1, 1.2)
    forig = (-1.5, 0.8, -0.6)
    fxyz = nrb.identity_header(fpix, forig)
    k, j, i = np.meshgrid(*[np.arange(n) for n in fdim[::-1]], indexing="ij")
    pts = [(i * fpix[0] + forig[0]).ravel(), (j * fpix[1] + forig[1]).ravel(), (k * fpix[2] + forig[2]).ravel()]
    flo = ndimage.map_coordinates(p.floating, [pts[2], pts[1], pts[0]], order=1, mode="constant", cval=0.0)
    return p.reference, (48, 44, 40), (1.0, 1.0, 1.0), nrb.identity_header((1.0, 1.0, 1.0)), \
        flo.reshape(fdim[::-1]).astype(np.float32), fdim, fpix, fxyz


def test_f3d2_registration_matches_reference(R):
    ref, rdim, rpix, rxyz, flo, fdim, fpix, fxyz = _pair()
    params = nrb.default_params(levels=2, max_iterations=20, bending_energy=0.005, spacing=(-5.0,), ref_bins=64,
                                flo_bins=64)
    gf, gb, (xf, xb), steps, wf, wb, r = nrb.f3d2_register_images(ref, rpix, rxyz, flo, fpix, fxyz, params)
    c_fw, c_bw, cdim, cxyz, ref_steps, st = R.f3d2_register(ref.ravel(), rdim, rpix, rxyz, flo.ravel(), fdim, fpix,
                                                            fxyz, 2, 20, 0.005, 0.0, 64, -5.0)
    print(f"final symmetric NMI b200 {r.final_nmi:.6f} reference {st[0]:.6f}; evaluations "
          f"{r.objective_evaluations}/{r.gradient_evaluations} vs {int(st[2])}/{int(st[3])}; steps {steps} vs "
          f"{ref_steps}; max |fw grid diff| {np.abs(c_fw - gf.ravel()).max():.3g} mm")
    assert list(cdim) == [gf.shape[3], gf.shape[2], gf.shape[1]] == list(r.cpp_dim)
    assert np.allclose(xf, cxyz, rtol=0, atol=1e-5)
    assert abs(r.final_nmi - st[0]) <= 5e-3 * st[0]
    assert r.final_nmi >= (1.0 - 1e-3) * st[0]
    # the result is symmetric: backward displacement = - forward displacement at every node
    ident = identity_grid(list(cdim), xf).reshape(gf.shape)
    ident_b = identity_grid(list(cdim), xb).reshape(gb.shape)
    assert np.allclose(gf - ident, -(gb - ident_b), atol=1e-4)
    assert wf.shape == ref.shape and wb.shape == flo.shape


def test_voxel_to_node_for_a_grid_not_aligned_with_the_image():
    """A rotated reference under an axis-aligned grid (the F3D2 situation): the workspace takes the
    general path (whole-volume convolution, node sampling through the full matrix). Against the
    oracle's restatement of Compute::ConvolveVoxelBasedMeasureGradient: within 1e-6 of the
    largest node value (the restatement itself is within 2e-7 of the reference here; the
    convolution sums run in another order)."""
    from tests.test_register_images_gpu import affine, rotation
    ensure_built()
    O = oracle.Restated()
    rdim, rpix = (26, 22, 18), (1.0, 1.1, 0.9)
    rxyz = affine(rotation(0.09, -0.05, 0.21), rpix, (-14.0, -12.5, -9.0))
    fdim, fpix = (24, 20, 20), (1.1, 1.0, 1.0)
    fxyz = affine(rotation(0.0, 0.1, -0.07), fpix, (-12.0, -11.0, -10.0))
    cdim, cpix = (10, 9, 8), (5.0, 5.0, 5.0)
    cxyz = nrb.identity_header(cpix, (-20.0, -18.0, -16.0))
    g = nrb.make_geometry(rdim, rpix, rxyz, fdim, fpix, fxyz, cdim, cpix, cxyz)
    vg = np.random.default_rng(71).normal(size=3 * int(np.prod(rdim))).astype(np.float32)
    _, ref = O.convolve_to_nodes(vg, rdim, rpix, np.array(g.ref_ijk, np.float32).reshape(4, 4), cdim, cpix, cxyz,
                                 np.array(g.flo_ijk, np.float32).reshape(4, 4), 0.7)
    ws = nrb.Workspace(g)
    node = torch.empty(3 * int(np.prod(cdim)), dtype=torch.float32, device="cuda")
    nrb.convolve_voxel_based_gradient(ws, dev(vg), node, 0.7)
    out = host(node)
    err = float(np.abs(out - ref).max())
    print(f"max |node - restatement| {err:.3g} (largest {np.abs(ref).max():.3g})")
    assert err <= 1e-6 * float(np.abs(ref).max())


def test_f3d2_registration_of_rotated_images_matches_reference(R):
    """The rotated pair of the image-geometry tests (reference and floating each under its own
    rotated sform, other dims and spacings): velocity grids axis-aligned in the world, so both
    images take the general voxel -> node path and the per-voxel flow evaluation."""
    from tests.test_register_images_gpu import OrientedPair
    o = OrientedPair()
    params = nrb.default_params(levels=2, max_iterations=20, bending_energy=0.005, spacing=(-5.0,), ref_bins=64,
                                flo_bins=64)
    gf, gb, (xf, xb), steps, wf, wb, r = nrb.f3d2_register_images(o.ref, o.rpix, o.rxyz, o.flo, o.fpix, o.fxyz, params)
    c_fw, c_bw, cdim, cxyz, ref_steps, st = R.f3d2_register(o.ref.ravel(), o.rdim, o.rpix, o.rxyz, o.flo.ravel(),
                                                            o.fdim, o.fpix, o.fxyz, 2, 20, 0.005, 0.0, 64, -5.0)
    print(f"rotated: final symmetric NMI b200 {r.final_nmi:.6f} reference {st[0]:.6f}; evaluations "
          f"{r.objective_evaluations}/{r.gradient_evaluations} vs {int(st[2])}/{int(st[3])}; steps {steps} vs "
          f"{ref_steps}")
    assert list(cdim) == [gf.shape[3], gf.shape[2], gf.shape[1]]
    assert np.allclose(xf, cxyz, rtol=0, atol=1e-5)
    assert abs(r.final_nmi - st[0]) <= 5e-3 * st[0]
    assert r.final_nmi >= (1.0 - 1e-3) * st[0]


def test_compose_refuses_aliased_fields():
    ensure_built()
    x = torch.zeros(3 * 8, dtype=torch.float32, device="cuda")
    with pytest.raises(nrb.NrbError):
        nrb.def_field_compose((2, 2, 2), np.eye(4, dtype=np.float32), x, x)


@pytest.mark.parametrize("update,amp,margin", [(True, 2.0, 1), (True, 25.0, 1), (False, 2.0, -2)])
def test_velocity_deformation_matches_the_restatement(update, amp, margin):
    """Against the C restatement (oracle/nrb_oracle.c): a grid that does not reach the whole
    field (margin -2) runs the border path of the flow kernel."""
    from tests.test_oracle_f3d2 import case
    ensure_built()
    O = oracle.Restated()
    fdim, fpix, fxyz, gdim, gpix, gxyz, vel = case(61, amp=amp, margin=margin)
    ref, rs = O.velocity_def_field(vel, gdim, gxyz, 6, update, fdim, fxyz)
    g = nrb.make_geometry(fdim, fpix, fxyz, fdim, fpix, fxyz, gdim, gpix, gxyz)
    d = torch.empty(3 * int(np.prod(fdim)), dtype=torch.float32, device="cuda")
    steps = nrb.get_def_field_from_velocity_grid(g, dev(vel), 6, d, update=update)
    assert steps == rs
    assert np.array_equal(host(d), ref)


def test_gradient_exponentiation_matches_the_restatement():
    from tests.test_oracle_f3d2 import case
    ensure_built()
    O = oracle.Restated()
    fdim, fpix, fxyz, gdim, gpix, gxyz, vel = case(63, amp=1.5)
    vg = np.random.default_rng(63).normal(0, 1, 3 * int(np.prod(fdim))).astype(np.float32)
    ref = O.exponentiate_gradient(fdim, fxyz, vel, gdim, gxyz, 7, vg)
    g = nrb.make_geometry(fdim, fpix, fxyz, fdim, fpix, fxyz, gdim, gpix, gxyz)
    t = dev(vg)
    nrb.exponentiate_gradient(g, dev(vel), 7, t)
    assert np.array_equal(host(t), ref)


def test_f3d2_file_request_writes_both_directions(tmp_path):
    """reg_f3d -vel on files: forward and backward grids and warped images, named as the
    reference's application names them, read back as the in-memory results."""
    ensure_built()
    ref, rdim, rpix, rxyz, flo, fdim, fpix, fxyz = _pair()
    params = nrb.default_params(levels=1, max_iterations=10, bending_energy=0.005, spacing=(-5.0,))
    nrb.write_image(tmp_path / "ref.nii.gz", ref, rpix, rxyz)
    nrb.write_image(tmp_path / "flo.nii", flo, fpix, fxyz)
    res = nrb.f3d2_register_files(tmp_path / "ref.nii.gz", tmp_path / "flo.nii", params, tmp_path / "cpp.nii.gz",
                                  tmp_path / "res.nii")
    gf, gb, (xf, xb), steps, wf, wb, r = nrb.f3d2_register_images(ref, rpix, rxyz, flo, fpix, fxyz, params)
    assert res.final_nmi == r.final_nmi and res.objective_evaluations == r.objective_evaluations
    c, _, cx = nrb.read_image(tmp_path / "cpp.nii.gz")
    cb, _, _ = nrb.read_image(tmp_path / "cpp_backward.nii.gz")
    assert np.array_equal(c, gf) and np.array_equal(cb, gb) and np.array_equal(cx, xf)
    w, _, _ = nrb.read_image(tmp_path / "res.nii")
    wbk, _, _ = nrb.read_image(tmp_path / "res_backward.nii")
    assert np.array_equal(w[0], wf, equal_nan=True) and np.array_equal(wbk[0], wb, equal_nan=True)
