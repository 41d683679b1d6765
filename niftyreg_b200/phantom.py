"""Seeded synthetic image pairs for the F3D workloads.

No public dataset is involved: every volume is generated from a seed. Each generator returns a
``Pair`` (reference, floating, voxel size) in float32, x-fastest ``[nz, ny, nx]`` order, the
memory layout NiftyReg's NIfTI volumes use.

* ``blobs_pair``  -- 12 Gaussian blobs (sigma U(3,8) voxels, amplitude U(200,1000)) and two
  ellipsoidal shells at 500 on a zero background, plus N(0,10) noise; the floating image is
  the reference warped by a cubic B-spline FFD (default 5-voxel control spacing, control
  displacements N(0,2) voxels) with trilinear interpolation.
* ``brain_pair``  -- a labelled 3-class phantom (class means 250/500/750, sigma 30) built from
  smooth random ellipsoids inside a head ellipsoid, times a smooth bias field in [0.9, 1.1];
  the floating image is warped by an FFD (5 mm spacing, N(0,3) mm displacements).
* ``ct_pair``     -- an HU phantom (air -1000, lung U(-900,-700), soft tissue N(40,20), bone
  U(300,1500) ellipsoids), floating warped by a 10 mm FFD with N(0,4) mm displacements.
"""
from __future__ import annotations

import dataclasses

import numpy as np
from scipy import ndimage

__all__ = ["Pair", "blobs_pair", "brain_pair", "ct_pair", "ffd_displacement", "warp_linear"]


@dataclasses.dataclass
class Pair:
    reference: np.ndarray  # float32 [nz, ny, nx]
    floating: np.ndarray   # float32 [nz, ny, nx]
    pixdim: tuple          # (dx, dy, dz) in mm

    @property
    def dim(self):
        nz, ny, nx = self.reference.shape
        return (nx, ny, nz)


def _bspline_weights(n: int, spacing_vox: float, ncp: int) -> np.ndarray:
    """Dense [n, ncp] matrix of cubic B-spline weights: voxel i uses nodes
    floor(i/s) .. floor(i/s)+3 of a grid whose node 0 sits one spacing before voxel 0."""
    w = np.zeros((n, ncp), dtype=np.float64)
    for i in range(n):
        t = i / spacing_vox
        k = int(np.floor(t))
        u = t - k
        b = ((1 - u) ** 3 / 6, (3 * u ** 3 - 6 * u ** 2 + 4) / 6,
             (-3 * u ** 3 + 3 * u ** 2 + 3 * u + 1) / 6, u ** 3 / 6)
        for a in range(4):
            if 0 <= k + a < ncp:
                w[i, k + a] = b[a]
    return w


def ffd_displacement(shape, spacing_vox, sigma_vox, rng) -> np.ndarray:
    """Random cubic B-spline FFD sampled on the voxel grid: returns [3, nz, ny, nx] voxel
    displacements (x, y, z components), control displacements N(0, sigma_vox)."""
    nz, ny, nx = shape
    sx, sy, sz = spacing_vox
    cx = int(np.ceil(nx / sx)) + 3
    cy = int(np.ceil(ny / sy)) + 3
    cz = int(np.ceil(nz / sz)) + 3
    wx = _bspline_weights(nx, sx, cx)
    wy = _bspline_weights(ny, sy, cy)
    wz = _bspline_weights(nz, sz, cz)
    out = np.empty((3, nz, ny, nx), dtype=np.float32)
    for c in range(3):
        cp = rng.normal(0.0, sigma_vox[c], size=(cz, cy, cx))
        t = np.tensordot(cp, wx, axes=([2], [1]))          # [cz, cy, nx]
        t = np.tensordot(t, wy, axes=([1], [1]))           # [cz, nx, ny]
        t = np.tensordot(t, wz, axes=([0], [1]))           # [nx, ny, nz]
        out[c] = np.transpose(t, (2, 1, 0)).astype(np.float32)
    return out


def warp_linear(img: np.ndarray, disp: np.ndarray) -> np.ndarray:
    """img(x + disp(x)) with trilinear interpolation and 0 outside the volume."""
    nz, ny, nx = img.shape
    zz, yy, xx = np.meshgrid(np.arange(nz, dtype=np.float32), np.arange(ny, dtype=np.float32),
                             np.arange(nx, dtype=np.float32), indexing="ij")
    coords = np.stack([zz + disp[2], yy + disp[1], xx + disp[0]])
    return ndimage.map_coordinates(img, coords, order=1, mode="constant", cval=0.0).astype(np.float32)


def _grid(shape):
    nz, ny, nx = shape
    return np.meshgrid(np.arange(nz, dtype=np.float32), np.arange(ny, dtype=np.float32),
                       np.arange(nx, dtype=np.float32), indexing="ij")


def blobs_pair(shape=(64, 64, 64), seed=0, spacing_vox=5.0, disp_sigma_vox=2.0) -> Pair:
    """Blob + shell phantom on a 1 mm grid; shape is (nz, ny, nx)."""
    rng = np.random.default_rng(seed)
    zz, yy, xx = _grid(shape)
    nz, ny, nx = shape
    ref = np.zeros(shape, dtype=np.float32)
    for _ in range(12):
        c = rng.uniform([0.2 * nz, 0.2 * ny, 0.2 * nx], [0.8 * nz, 0.8 * ny, 0.8 * nx])
        s = rng.uniform(3.0, 8.0)
        a = rng.uniform(200.0, 1000.0)
        ref += a * np.exp(-((zz - c[0]) ** 2 + (yy - c[1]) ** 2 + (xx - c[2]) ** 2) / (2 * s * s))
    for _ in range(2):
        c = rng.uniform([0.35 * nz, 0.35 * ny, 0.35 * nx], [0.65 * nz, 0.65 * ny, 0.65 * nx])
        r = rng.uniform([0.15 * nz, 0.15 * ny, 0.15 * nx], [0.35 * nz, 0.35 * ny, 0.35 * nx])
        d = np.sqrt(((zz - c[0]) / r[0]) ** 2 + ((yy - c[1]) / r[1]) ** 2 + ((xx - c[2]) / r[2]) ** 2)
        ref[np.abs(d - 1.0) < 0.08] = 500.0
    ref += rng.normal(0.0, 10.0, size=shape).astype(np.float32)
    disp = ffd_displacement(shape, (spacing_vox,) * 3, (disp_sigma_vox,) * 3, rng)
    flo = warp_linear(ref, disp)
    return Pair(ref.astype(np.float32), flo, (1.0, 1.0, 1.0))


def _head_labels(shape, rng, n_ellipsoids=24):
    zz, yy, xx = _grid(shape)
    nz, ny, nx = shape
    head = (((zz - nz / 2) / (0.45 * nz)) ** 2 + ((yy - ny / 2) / (0.45 * ny)) ** 2
            + ((xx - nx / 2) / (0.45 * nx)) ** 2) <= 1.0
    labels = np.where(head, 1, 0).astype(np.int8)
    for _ in range(n_ellipsoids):
        c = rng.uniform([0.25 * nz, 0.25 * ny, 0.25 * nx], [0.75 * nz, 0.75 * ny, 0.75 * nx])
        r = rng.uniform([0.05 * nz, 0.05 * ny, 0.05 * nx], [0.2 * nz, 0.2 * ny, 0.2 * nx])
        inside = (((zz - c[0]) / r[0]) ** 2 + ((yy - c[1]) / r[1]) ** 2 + ((xx - c[2]) / r[2]) ** 2) <= 1.0
        labels[inside & head] = rng.integers(1, 4)
    return labels, head


def brain_pair(shape=(182, 218, 182), seed=0, pixdim=(1.0, 1.0, 1.0), spacing_mm=5.0,
               disp_sigma_mm=3.0) -> Pair:
    """3-class brain-MR-like phantom; shape is (nz, ny, nx)."""
    rng = np.random.default_rng(seed)
    labels, head = _head_labels(shape, rng)
    means = np.array([0.0, 250.0, 500.0, 750.0], dtype=np.float32)
    ref = means[labels] + np.where(head, rng.normal(0.0, 30.0, size=shape), 0.0).astype(np.float32)
    zz, yy, xx = _grid(shape)
    nz, ny, nx = shape
    ph = rng.uniform(0, 2 * np.pi, size=3)
    bias = 1.0 + 0.1 * (np.cos(np.pi * zz / nz + ph[0]) * np.cos(np.pi * yy / ny + ph[1])
                        * np.cos(np.pi * xx / nx + ph[2]))
    ref = (ref * bias).astype(np.float32)
    sv = tuple(spacing_mm / p for p in pixdim)
    dv = tuple(disp_sigma_mm / p for p in pixdim)
    disp = ffd_displacement(shape, sv, dv, rng)
    flo = warp_linear(ref, disp)
    return Pair(ref, flo, tuple(float(p) for p in pixdim))


def ct_pair(shape=(320, 512, 512), seed=0, pixdim=(0.8, 0.8, 1.5), spacing_mm=10.0,
            disp_sigma_mm=4.0) -> Pair:
    """HU phantom of a CT-like chest; shape is (nz, ny, nx), pixdim is (dx, dy, dz)."""
    rng = np.random.default_rng(seed)
    zz, yy, xx = _grid(shape)
    nz, ny, nx = shape
    ref = np.full(shape, -1000.0, dtype=np.float32)
    body = (((yy - ny / 2) / (0.4 * ny)) ** 2 + ((xx - nx / 2) / (0.45 * nx)) ** 2) <= 1.0
    ref[body] = rng.normal(40.0, 20.0, size=int(body.sum())).astype(np.float32)
    for side in (-1, 1):
        lung = (((yy - ny / 2) / (0.25 * ny)) ** 2 + ((xx - nx / 2 - side * 0.2 * nx) / (0.15 * nx)) ** 2
                + ((zz - nz / 2) / (0.45 * nz)) ** 2) <= 1.0
        ref[lung] = rng.uniform(-900.0, -700.0, size=int(lung.sum())).astype(np.float32)
    for _ in range(10):
        c = rng.uniform([0.1 * nz, 0.2 * ny, 0.2 * nx], [0.9 * nz, 0.8 * ny, 0.8 * nx])
        r = rng.uniform([0.02 * nz, 0.01 * ny, 0.01 * nx], [0.1 * nz, 0.04 * ny, 0.04 * nx])
        bone = (((zz - c[0]) / r[0]) ** 2 + ((yy - c[1]) / r[1]) ** 2 + ((xx - c[2]) / r[2]) ** 2) <= 1.0
        ref[bone] = rng.uniform(300.0, 1500.0, size=int(bone.sum())).astype(np.float32)
    dx, dy, dz = pixdim
    disp = ffd_displacement(shape, (spacing_mm / dx, spacing_mm / dy, spacing_mm / dz),
                            (disp_sigma_mm / dx, disp_sigma_mm / dy, disp_sigma_mm / dz), rng)
    flo = warp_linear(ref, disp)
    return Pair(ref, flo, tuple(float(p) for p in pixdim))
