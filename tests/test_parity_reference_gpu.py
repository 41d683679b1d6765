"""The fused F3D evaluation on the GPU against the reference CPU path and the FP64 oracle.

Three CPU evaluations of the same seeded inputs (ref_evaluate.cpp, through the reference's own
functions) anchor each case:

* ``sse``    -- the reference's default build (oracle/_ref, SSE, single precision): the
                "reference CPU path" of the parity bars;
* ``fp64``   -- the FP64 oracle (oracle/_ref64, the reference's FLOAT64 instantiations);
* ``scalar`` -- the reference's build without SSE, single precision (oracle/_ref64): how far two
                builds of the reference itself sit apart.

Bars (each stated where it is asserted):

* deformation field: within 1e-4 voxel of the FP64 oracle, every voxel and component;
* NMI: within 1e-5 relative of the reference CPU path and of the FP64 oracle;
* bending energy: within 1e-6 relative;
* node gradient, relative L2: within 1e-4 of the FP64 oracle, or no further from it than the
  reference's own default build is (``max(1e-4, |sse - fp64|)``); and within 1e-4 of the
  reference CPU path wherever that path is itself within 1e-4 of the FP64 oracle.
  Single precision sets a floor here that no float implementation escapes: the spatial gradient
  of the trilinear interpolant jumps at voxel faces, so positions rounded to float (even
  correctly rounded ones) move a few voxels across a face relative to double positions. On the
  182x218x182 workload every float evaluation -- the reference's SSE build, its scalar build,
  this library -- lies 2e-4..4e-4 from the FP64 oracle and from each other, so there the bar
  against the reference CPU path is the triangle bound ``|gpu - fp64| + |sse - fp64|``;
* node gradient, largest single component: within max(2e-3, 2 x the reference's own
  |sse - fp64|) of the largest component (a gross-error cap with the same cause).

Every measured error is printed and, with NRB_PARITY_REPORT=<path>, appended to that file as one
JSON line per case.
"""
import json
import os

import numpy as np
import pytest

import niftyreg_b200 as nrb
import oracle
from niftyreg_b200 import phantom
from tests.helpers import Case, ensure_built, identity_grid, make_case, rescale

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

SIM_W, BE_W = 0.995, 0.005

SMALL = {
    "iso5": dict(),
    "spacing2": dict(shape=(16, 17, 19), spacing_vox=(2.0, 2.0, 2.0), seed=1),
    "aniso": dict(shape=(18, 30, 26), pixdim=(0.8, 0.8, 1.5), spacing_vox=(12.5, 12.5, 20.0 / 3.0), seed=2),
    "large_disp": dict(seed=6, disp=3.0),
    "bins132": dict(seed=5, bins=132),
    "medium": dict(shape=(64, 64, 64), seed=9, disp=2.0),
}


def full_case(kind):
    """The full-size workloads: 'brain182' = 182x218x182 at 1 mm, 5 mm grid, N(0, 3 mm) control
    displacements, 64 bins; 'ct512' = 512x512x320 at 0.8x0.8x1.5 mm, 10 mm grid, N(0, 4 mm),
    128 bins (132 internal)."""
    if kind == "brain182":
        shape, pix, spacing, sigma, bins, pair = (182, 218, 182), (1.0, 1.0, 1.0), 5.0, 3.0, 68, \
            phantom.brain_pair((182, 218, 182), seed=3)
    else:
        shape, pix, spacing, sigma, bins, pair = (320, 512, 512), (0.8, 0.8, 1.5), 10.0, 4.0, 132, \
            phantom.ct_pair((320, 512, 512), seed=4)
    nz, ny, nx = shape
    rdim = (nx, ny, nz)
    rxyz = nrb.identity_header(pix)
    cdim, cpix, cxyz = nrb.control_grid_header(rdim, pix, (spacing,) * 3)
    rng = np.random.default_rng(11)
    cpp = identity_grid(cdim, cxyz) + rng.normal(0, sigma, 3 * int(np.prod(cdim))).astype(np.float32)
    ref = rescale(pair.reference, 2, bins - 3).ravel()
    flo = rescale(pair.floating, 2, bins - 3).ravel()
    return Case(rdim, pix, rxyz, rdim, pix, rxyz, tuple(cdim), tuple(cpix), cxyz, ref, flo, cpp, bins)


@pytest.fixture(scope="module")
def refs():
    ensure_built()
    if not (oracle.ref_available() and oracle.ref64_available()):
        pytest.skip("reference libraries (oracle/_ref, oracle/_ref64) not built")
    sse, r64 = oracle.Ref(), oracle.Ref(oracle.REF64_SO)
    n = os.cpu_count() or 1
    sse.set_threads(n)
    r64.set_threads(n)
    return sse, r64


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def report(name, rec):
    print(f"[parity] {name}: " + ", ".join(f"{k} {v:.3g}" if isinstance(v, float) else f"{k} {v}"
                                           for k, v in rec.items()))
    path = os.environ.get("NRB_PARITY_REPORT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(dict(case=name, **rec)) + "\n")


def rel_l2(x, y):
    return float(np.linalg.norm(x - y) / np.linalg.norm(y))


def max_rel(x, y):
    return float(np.abs(x - y).max() / np.abs(y).max())


def check_case(name, c, refs, want_field=True):
    sse, r64 = refs
    args = (c.ref, c.rdim, c.rpix, c.rxyz, c.flo, c.fdim, c.fpix, c.fxyz, c.cpp, c.cdim, c.cpix, c.cxyz, c.bins,
            SIM_W, BE_W)
    a = sse.evaluate(*args)
    s = r64.evaluate(*args)
    d = r64.evaluate(*args, fp64=True, want_def=want_field)

    g = c.geometry()
    ws, nmi = nrb.Workspace(g), nrb.Nmi(c.bins, c.bins)
    rt, ft, ct = dev(c.ref), dev(c.flo), dev(c.cpp)
    o = nrb.f3d_objective(ws, nmi, rt, ft, ct, SIM_W, BE_W)
    vg = torch.empty(3 * c.nvox, dtype=torch.float32, device="cuda")
    node = torch.empty(3 * c.ncp, dtype=torch.float32, device="cuda")
    nrb.f3d_gradient(ws, nmi, rt, ft, ct, vg, node, SIM_W, BE_W)
    torch.cuda.synchronize()
    out = node.cpu().numpy().astype(np.float64)
    del vg
    rec = dict(nvox=c.nvox, bins=c.bins,
               nmi_gpu=o.nmi, nmi_sse=a["nmi"], nmi_fp64=d["nmi"],
               nmi_rel_vs_sse=abs(o.nmi - a["nmi"]) / a["nmi"], nmi_rel_vs_fp64=abs(o.nmi - d["nmi"]) / d["nmi"],
               be_rel_vs_sse=abs(o.be - a["be"]) / a["be"],
               node_l2_vs_sse=rel_l2(out, a["node"]), node_l2_vs_fp64=rel_l2(out, d["node"]),
               node_max_vs_sse=max_rel(out, a["node"]), node_max_vs_fp64=max_rel(out, d["node"]),
               sse_l2_vs_fp64=rel_l2(a["node"], d["node"]), sse_max_vs_fp64=max_rel(a["node"], d["node"]),
               scalar_l2_vs_fp64=rel_l2(s["node"], d["node"]), scalar_l2_vs_sse=rel_l2(s["node"], a["node"]),
               scalar_max_vs_sse=max_rel(s["node"], a["node"]))
    if want_field:
        dfield = torch.empty(3 * c.nvox, dtype=torch.float32, device="cuda")
        nrb.get_deformation_field(g, ct, dfield)
        torch.cuda.synchronize()
        df = dfield.cpu().numpy().astype(np.float64).reshape(3, -1)
        del dfield
        pix = np.asarray(c.rpix, np.float64)[:, None]
        rec["field_max_voxel_vs_fp64"] = float((np.abs(df - d["def"].reshape(3, -1)) / pix).max())
    report(name, rec)

    assert rec["nmi_rel_vs_sse"] <= 1e-5 and rec["nmi_rel_vs_fp64"] <= 1e-5
    assert rec["be_rel_vs_sse"] <= 1e-6
    # at least as close to the exact (FP64) node gradient as the reference's default build
    assert rec["node_l2_vs_fp64"] <= max(1e-4, rec["sse_l2_vs_fp64"]), rec
    if rec["sse_l2_vs_fp64"] <= 1e-4:
        assert rec["node_l2_vs_sse"] <= 1e-4, rec
    else:
        assert rec["node_l2_vs_sse"] <= rec["node_l2_vs_fp64"] + rec["sse_l2_vs_fp64"], rec
    assert rec["node_max_vs_fp64"] <= max(2e-3, 2 * rec["sse_max_vs_fp64"]), rec
    if want_field:
        assert rec["field_max_voxel_vs_fp64"] <= 1e-4, rec
    return rec


@pytest.mark.parametrize("name", list(SMALL))
def test_small_cases_against_reference_and_fp64(refs, name):
    check_case(name, make_case(**SMALL[name]), refs)


def test_brain_size_against_reference_and_fp64(refs):
    """182x218x182, 1 mm, 5 mm grid, 64 bins (the bench workload's finest level)."""
    check_case("brain182", full_case("brain182"), refs)


def test_ct_size_against_reference_and_fp64(refs):
    """512x512x320 at 0.8x0.8x1.5 mm, 10 mm grid, 128 bins: 83.9 M voxels, the 132x132
    histogram in shared memory."""
    check_case("ct512", full_case("ct512"), refs)
