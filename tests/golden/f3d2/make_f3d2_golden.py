"""Generates velocity.npz in this directory by running NiftyReg's own CPU code
(oracle/_ref/libnrref.so, compiled from the reference sources by `make -C oracle ref`) on small
seeded inputs of the F3D2 (reg_f3d2) velocity-field operations. The reference sources are only
needed to regenerate; the fixture is committed and the tests read it on any machine.

    python tests/golden/f3d2/make_f3d2_golden.py

Inputs: a 20x18x16 field (spacing 1.0 x 1.1 x 0.9 mm, origin (-3, 2, 1.5)), a 4 mm velocity grid
with N(0, 2 mm) node displacements (one node of margin; `vel_tight`: two nodes short of the field,
so the flow's sliding path runs), a voxel gradient, positions for the composition, and two grids
for the symmetrisation. Outputs of the reference's own functions:
  def6, def_upd, steps_upd  reg_spline_getDefFieldFromVelocityGrid (N = 6; N recomputed)
  def_tight                 the same on the grid short of the field (N = 6)
  composed                  reg_defField_compose (apply, pos)
  expgrad7                  Compute::ExponentiateGradient's sequence, N = 7
  sym_fw, sym_bw            Compute::SymmetriseVelocityFields
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from tests.test_oracle_f3d2 import case  # noqa: E402
from tests.helpers import identity_grid  # noqa: E402


def main():
    R = oracle.Ref()
    R.set_threads(1)
    fdim, fpix, fxyz, gdim, gpix, gxyz, vel = case(61)
    _, _, _, gdim_t, _, gxyz_t, vel_t = case(61, margin=-2)
    out = dict(fdim=np.array(fdim, np.int32), fpix=np.array(fpix, np.float32), fxyz=fxyz,
               gdim=np.array(gdim, np.int32), gpix=np.array(gpix, np.float32), gxyz=gxyz, vel=vel,
               gdim_tight=np.array(gdim_t, np.int32), gxyz_tight=gxyz_t, vel_tight=vel_t)
    out["def6"], _ = R.velocity_def_field(vel, gdim, gpix, gxyz, 6, False, fdim, fpix, fxyz)
    out["def_upd"], s = R.velocity_def_field(vel, gdim, gpix, gxyz, 6, True, fdim, fpix, fxyz)
    out["steps_upd"] = np.int32(s)
    out["def_tight"], _ = R.velocity_def_field(vel_t, gdim_t, gpix, gxyz_t, 6, False, fdim, fpix, fxyz)
    rng = np.random.default_rng(62)
    n = int(np.prod(fdim))
    k, j, i = np.meshgrid(*[np.arange(v) for v in fdim[::-1]], indexing="ij")
    vox = np.stack([i.ravel(), j.ravel(), k.ravel(), np.ones(n)])
    ident = (fxyz.astype(np.float64) @ vox)[:3].astype(np.float32).ravel()
    out["apply"] = (ident + rng.normal(0, 1.0, ident.size)).astype(np.float32)
    out["pos"] = (ident + rng.uniform(-5, 5, ident.size)).astype(np.float32)
    out["composed"] = R.def_compose(fdim, fpix, fxyz, out["apply"], out["pos"])
    out["vgrad"] = np.random.default_rng(63).normal(0, 1, 3 * n).astype(np.float32)
    out["expgrad7"] = R.exponentiate_gradient(fdim, fpix, fxyz, vel, gdim, gpix, gxyz, 7, out["vgrad"])
    bxyz = gxyz.copy()
    bxyz[:3, 3] += np.float32(0.75)
    rng = np.random.default_rng(64)
    out["bxyz"] = bxyz
    out["fw"] = (identity_grid(gdim, gxyz) + rng.normal(0, 2, vel.size)).astype(np.float32)
    out["bw"] = (identity_grid(gdim, bxyz) + rng.normal(0, 2, vel.size)).astype(np.float32)
    out["sym_fw"], out["sym_bw"] = R.symmetrise(gdim, gpix, gxyz, bxyz, out["fw"], out["bw"])
    np.savez_compressed(os.path.join(HERE, "velocity.npz"), **out)


if __name__ == "__main__":
    main()
