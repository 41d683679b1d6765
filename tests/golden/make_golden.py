"""Generates the golden fixtures of this directory by running NiftyReg's own CPU code
(oracle/_ref/libnrref.so, compiled from the reference sources by `make -C oracle ref`) on small
seeded inputs. The reference sources are only needed to regenerate; the fixtures are committed
and the tests read them on any machine.

    python tests/golden/make_golden.py

Each case file `<name>.npz` holds the inputs (images, grid, geometry) and the reference's outputs
for every step of the F3D objective/gradient path:
  def        reg_spline_getDeformationField (cubic B-spline, positions in mm)
  warped     reg_resampleImage, linear, NaN padding
  warped_nn, warped_cubic, warped_cubic_pad0
             reg_resampleImage, nearest / cubic spline (NaN padding) and cubic with padding 0
  wgrad      reg_getImageGradient, linear
  nmi, pro, logt, ent
             reg_nmi value, smoothed joint/marginal tables, log tables, entropies
  vgrad      reg_getVoxelBasedNmiGradient3d (weight 1)
  conv_x/y/z reg_tools_kernelConvolution, cubic, one axis at a time, on vgrad
  node       Compute::ConvolveVoxelBasedMeasureGradient (weight 0.995)
  be, be_grad
             reg_spline_approxBendingEnergy and its gradient (weight 0.005)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CASES = {
    # name: make_case keyword arguments ((nz, ny, nx) shapes, grid spacing in voxels)
    "iso": dict(shape=(12, 14, 16), spacing_vox=(4.0, 4.0, 4.0), seed=3, disp=1.2),
    "aniso": dict(shape=(10, 13, 17), pixdim=(1.2, 0.9, 1.5), spacing_vox=(3.0, 4.0, 3.0), seed=4, disp=1.0),
    "nan_bins36": dict(shape=(11, 12, 14), spacing_vox=(3.0, 3.0, 3.0), seed=5, bins=36, disp=1.0, nan_frac=0.03),
}


def generate(name, kw):
    import oracle
    from tests.helpers import make_case
    c = make_case(**kw)
    R = oracle.Ref()
    R.set_threads(1)
    d = R.deformation_field(c.cpp, c.cdim, c.cpix, c.cxyz, c.rdim, c.rpix, c.rxyz)
    w = R.resample(c.flo, c.fdim, c.fpix, c.fxyz, d, c.rdim, c.rpix, c.rxyz)
    w_nn = R.resample_order(c.flo, c.fdim, c.fpix, c.fxyz, d, c.rdim, c.rpix, c.rxyz, 0)
    w_cubic = R.resample_order(c.flo, c.fdim, c.fpix, c.fxyz, d, c.rdim, c.rpix, c.rxyz, 3)
    w_cubic0 = R.resample_order(c.flo, c.fdim, c.fpix, c.fxyz, d, c.rdim, c.rpix, c.rxyz, 3, pad=0.0)
    g = R.image_gradient(c.flo, c.fdim, c.fpix, c.fxyz, d, c.rdim, c.rpix, c.rxyz)
    nmi, pro, logt, ent = R.nmi_value(c.ref, w, c.rdim, c.bins, c.bins)
    vg = R.nmi_voxel_gradient(c.ref, w, g, c.rdim, c.bins, c.bins, 1.0)
    conv = {}
    for axis, key in enumerate(("conv_x", "conv_y", "conv_z")):
        conv[key] = R.kernel_convolution_cubic(vg, 3, c.rdim, c.rpix, c.cpix[axis], axis)
    _, node = R.convolve_to_nodes(vg, c.rdim, c.rpix, c.rxyz, c.fdim, c.fpix, c.fxyz, c.cdim, c.cpix, c.cxyz, 0.995)
    be = R.be_value(c.cpp, c.cdim, c.cpix, c.cxyz)
    be_grad = R.be_gradient(c.cpp, c.cdim, c.cpix, c.cxyz, 0.005)
    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"),
        rdim=np.array(c.rdim, np.int32), rpix=np.array(c.rpix, np.float32), rxyz=c.rxyz.astype(np.float32),
        fdim=np.array(c.fdim, np.int32), fpix=np.array(c.fpix, np.float32), fxyz=c.fxyz.astype(np.float32),
        cdim=np.array(c.cdim, np.int32), cpix=np.array(c.cpix, np.float32), cxyz=c.cxyz.astype(np.float32),
        bins=np.int32(c.bins), ref=c.ref, flo=c.flo, cpp=c.cpp,
        **{"def": d}, warped=w, warped_nn=w_nn, warped_cubic=w_cubic, warped_cubic_pad0=w_cubic0, wgrad=g, nmi=np.float64(nmi), pro=pro, logt=logt, ent=ent, vgrad=vg,
        node=node, be=np.float64(be), be_grad=be_grad, **conv)
    print(f"{name}: {c.rdim} grid {c.cdim} bins {c.bins} NMI {nmi:.10f} BE {be:.6g}")


if __name__ == "__main__":
    import oracle
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libnrref.so is missing: make -C oracle ref (needs the reference sources)")
    for name, kw in CASES.items():
        generate(name, kw)
