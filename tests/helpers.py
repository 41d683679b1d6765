"""Seeded test cases shared by the parity tests."""
from __future__ import annotations

import dataclasses
import os
import subprocess

import numpy as np

import niftyreg_b200 as nrb
from niftyreg_b200 import phantom

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def ensure_built():
    nrb.build()
    oracle_dir = os.path.join(ROOT, "oracle")
    if not os.path.exists(os.path.join(oracle_dir, "liboracle.so")):
        subprocess.check_call(["make", "-C", oracle_dir, "liboracle.so"], stdout=subprocess.DEVNULL)


class ArgBuffers:
    """Real buffers for the tests that check an entry point refuses bad arguments before any
    device work. With a CUDA device they are device allocations, so an entry point that launched
    a kernel before its checks would read valid memory and fail the test's assertion, never
    fault the device; without one no kernel can launch at all, and host buffers stand in."""

    def __init__(self, count=2, nbytes=1 << 16):
        import ctypes
        self._keep = []
        self.ptrs = []
        try:
            import torch
            cuda = torch.cuda.is_available()
        except Exception:
            cuda = False
        for _ in range(count):
            if cuda:
                t = torch.zeros(nbytes // 4, dtype=torch.float32, device="cuda")
                self._keep.append(t)
                self.ptrs.append(ctypes.c_void_p(t.data_ptr()))
            else:
                b = (ctypes.c_char * nbytes)()
                self._keep.append(b)
                self.ptrs.append(ctypes.c_void_p(ctypes.addressof(b)))

    def __getitem__(self, i):
        return self.ptrs[i]


@dataclasses.dataclass
class Case:
    rdim: tuple        # (nx, ny, nz)
    rpix: tuple
    rxyz: np.ndarray   # 4x4 voxel->mm
    fdim: tuple
    fpix: tuple
    fxyz: np.ndarray
    cdim: tuple
    cpix: tuple
    cxyz: np.ndarray
    ref: np.ndarray    # flat float32, rescaled to [2, bins-3]
    flo: np.ndarray
    cpp: np.ndarray    # flat float32, 3 planes
    bins: int          # internal bins (user + 4)

    @property
    def nvox(self):
        return int(np.prod(self.rdim))

    @property
    def ncp(self):
        return int(np.prod(self.cdim))

    def geometry(self):
        return nrb.make_geometry(self.rdim, self.rpix, self.rxyz, self.fdim, self.fpix, self.fxyz,
                                 self.cdim, self.cpix, self.cxyz)

    @property
    def ref_ijk(self):
        return np.linalg.inv(self.rxyz.astype(np.float64)).astype(np.float32)

    @property
    def flo_ijk(self):
        return np.linalg.inv(self.fxyz.astype(np.float64)).astype(np.float32)


def identity_grid(cdim, cxyz):
    """Node positions of an identity transformation, float arithmetic in the reference's order."""
    cx, cy, cz = cdim
    z, y, x = np.meshgrid(np.arange(cz, dtype=np.float32), np.arange(cy, dtype=np.float32),
                          np.arange(cx, dtype=np.float32), indexing="ij")
    m = cxyz.astype(np.float32)
    out = []
    for k in range(3):
        v = (m[k, 0] * x + m[k, 1] * y) + m[k, 2] * z
        out.append((v + m[k, 3]).ravel())
    return np.concatenate(out).astype(np.float32)


def rescale(img, lo, hi):
    img = img.astype(np.float32).copy()
    ok = np.isfinite(img)
    mn, mx = img[ok].min(), img[ok].max()
    v = (img.astype(np.float64) - float(mn)) / float(mx - mn) * (hi - lo) + lo
    img[ok] = v[ok].astype(np.float32)
    return img


def make_case(shape=(20, 24, 28), pixdim=(1.0, 1.0, 1.0), spacing_vox=(5.0, 5.0, 5.0), seed=0, bins=68,
              disp=1.5, flo_shape=None, flo_pixdim=None, nan_frac=0.0):
    """shape is (nz, ny, nx). The grid is built as reg_createControlPointGrid does."""
    rng = np.random.default_rng(seed)
    pair = phantom.blobs_pair(shape, seed=seed)
    nz, ny, nx = shape
    rdim = (nx, ny, nz)
    rpix = tuple(float(p) for p in pixdim)
    rxyz = nrb.identity_header(rpix)
    flo = pair.floating
    fdim, fpix = rdim, rpix
    if flo_shape is not None:
        flo = phantom.blobs_pair(flo_shape, seed=seed + 100).floating
        fdim = (flo_shape[2], flo_shape[1], flo_shape[0])
        fpix = tuple(float(p) for p in (flo_pixdim or pixdim))
    fxyz = nrb.identity_header(fpix)
    spacing_mm = [s * p for s, p in zip(spacing_vox, rpix)]
    cdim, cpix, cxyz = nrb.control_grid_header(rdim, rpix, spacing_mm)
    cpp = identity_grid(cdim, cxyz) + rng.normal(0, disp, 3 * int(np.prod(cdim))).astype(np.float32)
    ref = rescale(pair.reference, 2, bins - 3).ravel()
    flo = rescale(flo, 2, bins - 3).ravel()
    if nan_frac > 0:
        ref[rng.random(ref.size) < nan_frac] = np.nan
    return Case(rdim, rpix, rxyz, tuple(fdim), fpix, fxyz, tuple(cdim), tuple(cpix), cxyz, ref, flo,
                cpp.astype(np.float32), bins)
