"""The CUDA path, through the C ABI, against the golden fixtures that NiftyReg's own CPU code
produced (tests/golden/make_golden.py). Each step is fed the reference's inputs for that step.

Tolerances: deformation field within 1e-4 voxel; warped intensities and
spatial gradients within 1e-4 on [2, bins-3]-scaled images with identical NaN patterns; NMI
within 1e-10 relative and tables within 1e-10 relative (integer counts, FP64 tables); voxel
gradient within 1e-5 of its largest magnitude; one-axis convolutions within 1e-5 of the largest
magnitude; node gradient within 1e-5 relative L2 on the reference's own voxel gradient; bending
energy within 1e-6 relative and its gradient within 1e-6 of the largest magnitude.
"""
import glob
import os

import numpy as np
import pytest

import niftyreg_b200 as nrb
from tests.helpers import ensure_built

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.fixture(params=CASES, ids=[os.path.basename(c)[:-4] for c in CASES])
def gold(request):
    ensure_built()
    g = dict(np.load(request.param))
    g["geom"] = nrb.make_geometry(tuple(g["rdim"]), tuple(g["rpix"]), g["rxyz"], tuple(g["fdim"]), tuple(g["fpix"]),
                                  g["fxyz"], tuple(g["cdim"]), tuple(g["cpix"]), g["cxyz"])
    return g


def test_deformation_field(gold):
    g = gold
    out = torch.empty(g["def"].size, dtype=torch.float32, device="cuda")
    nrb.get_deformation_field(g["geom"], dev(g["cpp"]), out)
    err = np.abs(host(out) - g["def"]).reshape(3, -1) / g["rpix"].reshape(3, 1)
    assert err.max() <= 1e-4


def test_resample_and_gradient(gold):
    g = gold
    d, flo = dev(g["def"]), dev(g["flo"])
    w = torch.empty(g["warped"].size, dtype=torch.float32, device="cuda")
    nrb.resample_image(g["geom"], flo, d, w)
    out = host(w)
    assert np.array_equal(np.isnan(out), np.isnan(g["warped"]))
    ok = ~np.isnan(out)
    assert np.abs(out[ok] - g["warped"][ok]).max() <= 1e-4
    gr = torch.empty(g["wgrad"].size, dtype=torch.float32, device="cuda")
    nrb.get_image_gradient(g["geom"], flo, d, gr)
    assert np.abs(host(gr) - g["wgrad"]).max() <= 1e-4


def test_nmi_and_voxel_gradient(gold):
    g = gold
    b = int(g["bins"])
    nmi = nrb.Nmi(b, b)
    v = nrb.nmi_value(nmi, g["geom"], dev(g["ref"]), dev(g["warped"]))
    assert abs(v - g["nmi"]) <= 1e-10 * g["nmi"]
    pro, logt, ent = nmi.tables()
    np.testing.assert_allclose(pro, g["pro"], rtol=1e-10, atol=1e-15)
    np.testing.assert_allclose(ent, g["ent"], rtol=1e-10)
    vg = torch.zeros(g["vgrad"].size, dtype=torch.float32, device="cuda")
    nrb.nmi_voxel_gradient(nmi, g["geom"], dev(g["ref"]), dev(g["warped"]), dev(g["wgrad"]), vg, 1.0)
    assert np.abs(host(vg) - g["vgrad"]).max() <= 1e-5 * np.abs(g["vgrad"]).max()


def test_kernel_convolution(gold):
    g = gold
    for axis, key in enumerate(("conv_x", "conv_y", "conv_z")):
        t = dev(g["vgrad"])
        nrb.kernel_convolution_cubic(t, 3, tuple(g["rdim"]), tuple(g["rpix"]), float(g["cpix"][axis]), axis)
        out, ref = host(t), g[key]
        assert np.array_equal(np.isnan(out), np.isnan(ref))
        ok = np.isfinite(ref)
        assert np.abs(out[ok] - ref[ok]).max() <= 1e-5 * np.abs(ref[ok]).max()


def test_convolve_to_nodes(gold):
    g = gold
    ws = nrb.Workspace(g["geom"])
    node = torch.empty(g["node"].size, dtype=torch.float32, device="cuda")
    nrb.convolve_voxel_based_gradient(ws, dev(g["vgrad"]), node, 0.995)
    out = host(node)
    assert np.linalg.norm(out - g["node"]) <= 1e-5 * np.linalg.norm(g["node"])


def test_bending_energy(gold):
    g = gold
    ws = nrb.Workspace(g["geom"])
    be = nrb.approx_bending_energy(ws, dev(g["cpp"]))
    assert abs(be - g["be"]) <= 1e-6 * abs(g["be"])
    grad = torch.zeros(g["be_grad"].size, dtype=torch.float32, device="cuda")
    nrb.approx_bending_energy_gradient(ws, dev(g["cpp"]), grad, 0.005)
    assert np.abs(host(grad) - g["be_grad"]).max() <= 1e-6 * np.abs(g["be_grad"]).max()
