"""NiftyReg's own reg_f3d<float>::Run on the B200 platform (niftyreg_b200/platform): the
reference's registration library built from its sources with the B200 Platform classes in place
of reg-lib/Platform.cpp. reg_f3d, the conjugate-gradient optimiser and the pyramid driver are the
reference's; every Compute, NMI and optimiser step of the B200 platform is one call of the C ABI.

CPU (no GPU): the library loads and exports what include/niftyreg_b200_platform.h declares, and
its CPU platform (the registry's CPU branch, the reference's own classes) registers bit for bit
like the reference library built by the oracle recipe.

GPU: the B200 platform against the CPU platform of the same library, same inputs:
- the first objective evaluation (max_iterations 0, one and two pyramid levels): NMI within 1e-5
  relative (the float warp and histogram against the reference's SSE float path);
- a full 64^3 registration (1 level, 100 iterations, BE 0.005, 64 bins, 5-voxel grid): the two
  follow the same optimiser branches until a line-search comparison flips on a last-bit
  difference, so the bar is on the end point, as for the fused path: final NMI within 5e-3
  relative, and not worse than the CPU platform's by more than 1e-3 relative;
- the platform's device work runs in libniftyreg_b200.so's kernels (launch counter);
- a setting outside the platform's scope raises the reference's fatal error instead of running
  on the host.
"""
import os
import re

import numpy as np
import pytest

import niftyreg_b200 as nrb
import oracle
from niftyreg_b200 import phantom
from tests.helpers import ROOT, ensure_built

needs_platform = pytest.mark.skipif(not nrb.platform_available(),
                                    reason="niftyreg_b200/platform library not built (needs the NiftyReg sources)")


@pytest.fixture(scope="module")
def small():
    return phantom.blobs_pair((32, 36, 40), seed=3)


@needs_platform
def test_platform_library_exports_declared_symbols():
    ensure_built()
    text = open(os.path.join(ROOT, "include", "niftyreg_b200_platform.h")).read()
    names = set(re.findall(r"\b(nrb_platform_[a-z_0-9]+)\s*\(", text))
    assert names == {"nrb_platform_last_error", "nrb_platform_f3d_register"}
    L = nrb.platform_lib()
    for n in names:
        assert hasattr(L, n), n


@needs_platform
def test_platform_refuses_bad_arguments(small):
    with pytest.raises(nrb.NrbError, match="levels"):
        nrb.platform_register(small.reference, small.floating, small.pixdim, platform=nrb.PLATFORM_CPU, levels=0)
    with pytest.raises(nrb.NrbError, match="unknown platform"):
        nrb.platform_register(small.reference, small.floating, small.pixdim, platform=7)


@needs_platform
def test_cpu_platform_equals_reference_library(small):
    """The registry's CPU branch is the reference's CPU platform: same grid, NMI and counts as
    the reference library the oracle recipe builds from the same sources with the same flags."""
    if not oracle.ref_available():
        pytest.skip("oracle/_ref/libnrref.so not built")
    R = oracle.Ref()
    R.set_threads(4)
    xyz = nrb.identity_header(small.pixdim)
    cpp, res = nrb.platform_register(small.reference, small.floating, small.pixdim, xyz, platform=nrb.PLATFORM_CPU,
                                     levels=2, max_iterations=15, bending_energy=0.005, spacing=-5.0, bins=32)
    c_ref, cdim, st = R.f3d_register(small.reference.ravel(), small.floating.ravel(), small.dim, small.pixdim, xyz,
                                     2, 15, 0.005, 0.0, 32, -5.0)
    assert list(cdim) == list(res.cpp_dim)
    assert np.array_equal(cpp.ravel(), c_ref)
    assert res.final_nmi == st[0]
    assert (res.objective_evaluations, res.gradient_evaluations) == (int(st[2]), int(st[3]))


# ---------------------------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------------------------
@pytest.fixture(scope="module")
def pair():
    ensure_built()
    import torch
    torch.cuda.set_device(0)
    return phantom.blobs_pair((64, 64, 64), seed=1)


def _identity_spread(pair):
    """|NMI(SSE build) - NMI(FP64 oracle)| / NMI(FP64) of one evaluation at the identity grid,
    NaN padding: how far the reference's own builds sit apart on this pair at the start."""
    R, R64 = oracle.Ref(), oracle.Ref(oracle.REF64_SO)
    xyz = nrb.identity_header(pair.pixdim)
    cpp, cdim, cpix, cxyz = R.create_control_point_grid(pair.dim, pair.pixdim, xyz, (5.0,) * 3)
    args = (pair.reference.ravel(), pair.dim, pair.pixdim, xyz, pair.floating.ravel(), pair.dim, pair.pixdim, xyz,
            cpp, cdim, cpix, cxyz, 68, 0.995, 0.005)
    sse, f64 = R.evaluate(*args)["nmi"], R64.evaluate(*args, fp64=True)["nmi"]
    return abs(sse - f64) / f64


@pytest.mark.gpu
@needs_platform
@pytest.mark.parametrize("levels", [1, 2])
@pytest.mark.parametrize("padding", [0.0, float("nan")])
def test_first_evaluation_matches_cpu_platform(pair, levels, padding):
    """The objective at the identity grid. With padding 0 every voxel counts and the NMI agrees
    within 1e-5 relative. With NaN padding a voxel on a far face of the volume counts only when
    its computed position falls below the face, so its last trilinear tap stays inside: at the
    identity the exact position lies on the face, and which side a build's rounding puts it on
    decides the voxel (the reference's SSE build puts 10% of them below, its FP64 build half of
    them; this library's positions are exact there). The bar is then the reference's own
    SSE-to-FP64 spread at the identity on this pair, or 1e-5 if that is larger."""
    if np.isnan(padding) and not (oracle.ref_available() and oracle.ref64_available()):
        pytest.skip("reference builds (oracle/_ref, oracle/_ref64) not built")
    kw = dict(levels=levels, max_iterations=0, bending_energy=0.005, spacing=-5.0, bins=64, padding=padding)
    c_cpu, r_cpu = nrb.platform_register(pair.reference, pair.floating, pair.pixdim, platform=nrb.PLATFORM_CPU, **kw)
    c_b2, r_b2 = nrb.platform_register(pair.reference, pair.floating, pair.pixdim, platform=nrb.PLATFORM_B200, **kw)
    rel = abs(r_b2.final_nmi - r_cpu.final_nmi) / r_cpu.final_nmi
    bar = 1e-5 if padding == 0.0 else max(1e-5, _identity_spread(pair))
    print(f"[platform] first evaluation, {levels} level(s), padding {padding}: NMI B200 {r_b2.final_nmi:.9f} "
          f"CPU {r_cpu.final_nmi:.9f}, relative {rel:.3g} (bar {bar:.3g})")
    assert r_b2.objective_evaluations == r_cpu.objective_evaluations == levels
    assert rel <= bar
    assert np.array_equal(c_b2, c_cpu)  # no step taken: the grids are the refined identity grids


@pytest.mark.gpu
@needs_platform
def test_registration_matches_cpu_platform(pair):
    kw = dict(levels=1, max_iterations=100, bending_energy=0.005, spacing=-5.0, bins=64)
    n0 = nrb.kernel_launch_count()
    c_b2, r_b2 = nrb.platform_register(pair.reference, pair.floating, pair.pixdim, platform=nrb.PLATFORM_B200, **kw)
    launches = nrb.kernel_launch_count() - n0
    c_cpu, r_cpu = nrb.platform_register(pair.reference, pair.floating, pair.pixdim, platform=nrb.PLATFORM_CPU, **kw)
    print(f"[platform] 64^3 registration: NMI B200 {r_b2.final_nmi:.8f} ({r_b2.seconds:.2f} s, "
          f"{r_b2.objective_evaluations}/{r_b2.gradient_evaluations} evaluations, {launches} kernel launches) "
          f"CPU {r_cpu.final_nmi:.8f} ({r_cpu.seconds:.2f} s, {r_cpu.objective_evaluations}/"
          f"{r_cpu.gradient_evaluations}); max |cpp diff| {np.abs(c_b2 - c_cpu).max():.4g} mm")
    assert launches >= 4 * r_b2.objective_evaluations  # deformation, warp, histogram, finalize per evaluation
    assert abs(r_b2.final_nmi - r_cpu.final_nmi) <= 5e-3 * r_cpu.final_nmi
    assert r_b2.final_nmi >= (1.0 - 1e-3) * r_cpu.final_nmi


@pytest.mark.gpu
@needs_platform
def test_ct_like_two_levels_matches_cpu_platform():
    """Anisotropic voxels (0.8 x 0.8 x 1.5 mm), a 10 mm grid, two levels with grid refinement
    between them: the reference driver on both platforms, same end-point bar."""
    ensure_built()
    p = phantom.ct_pair((40, 72, 64), seed=2)
    kw = dict(levels=2, max_iterations=30, bending_energy=0.001, spacing=10.0, bins=64)
    c_b2, r_b2 = nrb.platform_register(p.reference, p.floating, p.pixdim, platform=nrb.PLATFORM_B200, **kw)
    c_cpu, r_cpu = nrb.platform_register(p.reference, p.floating, p.pixdim, platform=nrb.PLATFORM_CPU, **kw)
    print(f"[platform] CT-like 2 levels: NMI B200 {r_b2.final_nmi:.8f} CPU {r_cpu.final_nmi:.8f}; evaluations "
          f"{r_b2.objective_evaluations}/{r_b2.gradient_evaluations} vs {r_cpu.objective_evaluations}/"
          f"{r_cpu.gradient_evaluations}")
    assert c_b2.shape == c_cpu.shape
    assert abs(r_b2.final_nmi - r_cpu.final_nmi) <= 5e-3 * r_cpu.final_nmi
    assert r_b2.final_nmi >= (1.0 - 1e-3) * r_cpu.final_nmi


@pytest.mark.gpu
@needs_platform
def test_platform_equals_fused_path_start(pair):
    """The platform's step-by-step calls and the fused registration driver start from the same
    first evaluation."""
    _, r_b2 = nrb.platform_register(pair.reference, pair.floating, pair.pixdim, platform=nrb.PLATFORM_B200,
                                    levels=1, max_iterations=0, bending_energy=0.005, spacing=-5.0, bins=64)
    _, r_fused = nrb.register_host(pair.reference, pair.floating, pair.pixdim,
                                   nrb.default_params(levels=1, max_iterations=0, bending_energy=0.005,
                                                      spacing=(-5.0,), ref_bins=64, flo_bins=64))
    assert abs(r_b2.final_nmi - r_fused.final_nmi) <= 1e-6 * r_fused.final_nmi


@pytest.mark.gpu
@needs_platform
def test_out_of_scope_setting_raises(pair):
    with pytest.raises(nrb.NrbError, match="not available on the B200 platform"):
        nrb.platform_register(pair.reference, pair.floating, pair.pixdim, platform=nrb.PLATFORM_B200, levels=1,
                              max_iterations=5, linear_energy=0.01)
