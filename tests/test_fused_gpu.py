"""The fused F3D evaluations against the oracle pipeline, plus determinism and full-size
properties.

Tolerances: NMI within 1e-5 relative; bending energy within 1e-6 relative; node gradient
within NODE_L2 in relative L2 norm, and no component off by more than NODE_MAX of the largest
magnitude (a gross-error cap). The node-gradient bounds are set by the reference itself: the
spatial gradient of a trilinear interpolant jumps at voxel faces, so a 1e-5 mm change of a
warped position can move one voxel's contribution across the jump. The reference's own SSE
build and its scalar arithmetic (the oracle) differ by 2.5e-5..9e-5 (L2) and 3e-5..1.3e-4
(max) on the small cases and by 1.2e-4 (L2) / 1.7e-3 (max) on the 182x218x182 case. Repeated
evaluations must be bit-identical (integer histograms, fixed-order FP64 reductions).
"""
import math

import numpy as np
import pytest

import niftyreg_b200 as nrb
import oracle
from niftyreg_b200 import phantom
from tests.helpers import ensure_built, identity_grid, make_case, rescale

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

CASES = {
    "iso5": dict(),
    "spacing2": dict(shape=(16, 17, 19), spacing_vox=(2.0, 2.0, 2.0), seed=1),
    "aniso": dict(shape=(18, 30, 26), pixdim=(0.8, 0.8, 1.5), spacing_vox=(12.5, 12.5, 20.0 / 3.0), seed=2),
    "large_disp": dict(seed=6, disp=3.0),
    "bins132": dict(seed=5, bins=132),
}
SIM_W, BE_W = 0.995, 0.005
NODE_L2, NODE_MAX = 3e-4, 5e-2


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


def oracle_objective(O, c):
    dfield = O.deformation_field(c.cpp, c.cdim, c.cpix, c.rdim, c.rpix)
    warped = O.resample(c.flo, c.fdim, c.flo_ijk, dfield, c.rdim)
    v, _, log, ent = O.nmi_value(c.ref, warped, c.bins, c.bins)
    be = O.be_value(c.cpp, c.cdim)
    return v, be, dfield, warped, log, ent


def oracle_gradient(O, c):
    _, _, dfield, warped, log, ent = oracle_objective(O, c)
    wgrad = O.image_gradient(c.flo, c.fdim, c.flo_ijk, dfield, c.rdim)
    vg = O.nmi_voxel_gradient(c.ref, warped, wgrad, c.bins, c.bins, log, ent, 1.0)
    _, node = O.convolve_to_nodes(vg, c.rdim, c.rpix, c.ref_ijk, c.cdim, c.cpix, c.cxyz, c.flo_ijk, SIM_W)
    return O.be_gradient(c.cpp, c.cdim, c.cxyz, BE_W, grad_init=node)


def test_fused_objective(O, case):
    c = case
    g = c.geometry()
    ws, nmi = nrb.Workspace(g), nrb.Nmi(c.bins, c.bins)
    o = nrb.f3d_objective(ws, nmi, dev(c.ref), dev(c.flo), dev(c.cpp), SIM_W, BE_W)
    v, be, *_ = oracle_objective(O, c)
    assert abs(o.nmi - v) <= 1e-5 * abs(v), (o.nmi, v)
    assert abs(o.be - be) <= 1e-6 * abs(be)
    assert abs(o.objective - (SIM_W * o.nmi - BE_W * o.be)) <= 1e-12


def test_fused_gradient(O, case):
    c = case
    g = c.geometry()
    ws, nmi = nrb.Workspace(g), nrb.Nmi(c.bins, c.bins)
    vg = torch.empty(3 * c.nvox, dtype=torch.float32, device="cuda")
    node = torch.full((3 * c.ncp,), 7.0, dtype=torch.float32, device="cuda")
    nrb.f3d_gradient(ws, nmi, dev(c.ref), dev(c.flo), dev(c.cpp), vg, node, SIM_W, BE_W)
    ref = oracle_gradient(O, c)
    out = host(node)
    scale = np.abs(ref).max()
    err = np.abs(out - ref).max()
    l2 = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert l2 <= NODE_L2, f"node gradient L2 error {l2:.3g}"
    assert err <= NODE_MAX * scale, f"node gradient error {err / scale:.3g} of max"


def test_repeatable_bitwise():
    c = make_case(shape=(40, 44, 48), seed=21, disp=2.0)
    g = c.geometry()
    ws, nmi = nrb.Workspace(g), nrb.Nmi(c.bins, c.bins)
    ref, flo, cpp = dev(c.ref), dev(c.flo), dev(c.cpp)
    a = nrb.f3d_objective(ws, nmi, ref, flo, cpp, SIM_W, BE_W)
    b = nrb.f3d_objective(ws, nmi, ref, flo, cpp, SIM_W, BE_W)
    assert a.nmi == b.nmi and a.be == b.be and list(a.entropy) == list(b.entropy)
    vg = torch.empty(3 * c.nvox, dtype=torch.float32, device="cuda")
    n1 = torch.empty(3 * c.ncp, dtype=torch.float32, device="cuda")
    n2 = torch.empty_like(n1)
    nrb.f3d_gradient(ws, nmi, ref, flo, cpp, vg, n1, SIM_W, BE_W)
    nrb.f3d_gradient(ws, nmi, ref, flo, cpp, vg, n2, SIM_W, BE_W)
    assert torch.equal(n1, n2)


@pytest.mark.parametrize("shape", [(40, 44, 48), (91, 109, 91)])
def test_fused_equals_staged_pipeline_bitwise(shape):
    """The fused objective (16-row items, z-chunks sized for its occupancy) and the staged
    pipeline (deformation field with 4-row items, resampling, histogram) decompose the volume
    differently; a voxel's position must not depend on that, so both give the same histogram,
    hence bit-identical NMI tables."""
    c = make_case(shape=shape, seed=23, disp=2.0)
    g = c.geometry()
    ref, flo, cpp = dev(c.ref), dev(c.flo), dev(c.cpp)
    ws, nmi_a, nmi_b = nrb.Workspace(g), nrb.Nmi(c.bins, c.bins), nrb.Nmi(c.bins, c.bins)
    fused = nrb.f3d_objective(ws, nmi_a, ref, flo, cpp, 1.0, 0.0)
    d = torch.empty(3 * c.nvox, dtype=torch.float32, device="cuda")
    w = torch.empty(c.nvox, dtype=torch.float32, device="cuda")
    nrb.get_deformation_field(g, cpp, d)
    nrb.resample_image(g, flo, d, w)
    staged = nrb.nmi_value(nmi_b, g, ref, w)
    assert fused.nmi == staged
    pa, la, ea = nmi_a.tables()
    pb, lb, eb = nmi_b.tables()
    assert np.array_equal(pa, pb) and np.array_equal(la, lb)


def test_zero_similarity_weight():
    c = make_case(seed=22)
    ws, nmi = nrb.Workspace(c.geometry()), nrb.Nmi(c.bins, c.bins)
    o = nrb.f3d_objective(ws, nmi, dev(c.ref), dev(c.flo), dev(c.cpp), 0.0, 1.0)
    assert o.nmi == 0.0 and o.objective == -o.be


def test_full_size_against_oracle(O):
    """The brain-MR-sized workload (182x218x182, 1 mm, 5 mm grid, N(0,3 mm) control
    displacements): fused objective and gradient against the full oracle pipeline, and
    bit-identical repeats."""
    shape = (182, 218, 182)
    pair = phantom.brain_pair(shape, seed=3)
    nz, ny, nx = shape
    rdim, rpix = (nx, ny, nz), (1.0, 1.0, 1.0)
    rxyz = nrb.identity_header(rpix)
    cdim, cpix, cxyz = nrb.control_grid_header(rdim, rpix, (5.0, 5.0, 5.0))
    rng = np.random.default_rng(3)
    cpp = identity_grid(cdim, cxyz) + rng.normal(0, 3.0, 3 * int(np.prod(cdim))).astype(np.float32)
    ref = rescale(pair.reference, 2, 65).ravel()
    flo = rescale(pair.floating, 2, 65).ravel()
    from tests.helpers import Case
    c = Case(rdim, rpix, rxyz, rdim, rpix, rxyz, tuple(cdim), tuple(cpix), cxyz, ref, flo, cpp, 68)
    g = c.geometry()
    ws, nmi = nrb.Workspace(g), nrb.Nmi(68, 68)
    rt, ft, ct = dev(ref), dev(flo), dev(cpp)
    a = nrb.f3d_objective(ws, nmi, rt, ft, ct, SIM_W, BE_W)
    b = nrb.f3d_objective(ws, nmi, rt, ft, ct, SIM_W, BE_W)
    assert a.nmi == b.nmi and a.be == b.be
    v, be, *_ = oracle_objective(O, c)
    assert abs(a.nmi - v) <= 1e-5 * v
    assert abs(a.be - be) <= 1e-6 * be
    vg = torch.empty(3 * c.nvox, dtype=torch.float32, device="cuda")
    node = torch.empty(3 * c.ncp, dtype=torch.float32, device="cuda")
    nrb.f3d_gradient(ws, nmi, rt, ft, ct, vg, node, SIM_W, BE_W)
    ref_node = oracle_gradient(O, c)
    out = host(node)
    assert np.linalg.norm(out - ref_node) <= NODE_L2 * np.linalg.norm(ref_node)
    assert np.abs(out - ref_node).max() <= NODE_MAX * np.abs(ref_node).max()
