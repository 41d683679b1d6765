"""Test infrastructure: the CPU oracle for the F3D objective-and-gradient path.

Two CPU implementations sit here, both used only as checkers (by ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``), never by the product:

* ``restated`` -- ``liboracle.so`` built from ``nrb_oracle.c``, a plain-C restatement of the
  reference algorithm, each function citing the reference file:line it follows;
* ``ref``      -- ``_ref/libnrref.so``, the reference NiftyReg CPU library itself, compiled from
  its own sources by ``oracle/Makefile`` (target ``ref``) plus the adapters ``ref_shim.cpp`` and
  ``ref_evaluate.cpp``;
* ``ref64``    -- ``_ref64/libnrref64.so``, the same sources built without the SSE path (target
  ``ref64``): the FP64 oracle (``evaluate(..., fp64=True)`` runs the reference's FLOAT64
  instantiations) and the reference's scalar single-precision build.

Parity of the restatement is pinned against ``ref`` and against the reference's own
known-answer tests (see ``tests/test_oracle_pins.py``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATED_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libnrref.so")
REF64_SO = os.path.join(HERE, "_ref64", "libnrref64.so")
REFCUDA_SO = os.path.join(HERE, "_refcuda", "libnrref_cuda.so")

_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _f(a):
    return a.ctypes.data_as(_fp) if a is not None else None


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def _i3(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.int32))


def _f3(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.float32))


def _m(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.float32).reshape(16))


def build_restated():
    if not os.path.exists(RESTATED_SO):
        subprocess.check_call(["make", "-C", HERE, "liboracle.so"], stdout=subprocess.DEVNULL)


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref64_available() -> bool:
    return os.path.exists(REF64_SO)


def refcuda_available() -> bool:
    return os.path.exists(REFCUDA_SO)


def refcuda_register(ref, flo, dim, pix, xyz, levels, maxit, be, le, bins, spacing, verbose=False):
    """reg_f3d<float>::Run on the reference's own CUDA platform (oracle/_refcuda, its reg-lib/cuda
    sources built for sm_100a): (cpp, cdim, stats) with stats as ``Ref.f3d_register``'s. Needs a
    GPU; the library creates its own CUDA context on the device it picks."""
    lib = ctypes.CDLL(REFCUDA_SO)
    params = np.array([levels, maxit, be, le, bins, spacing, 1 if verbose else 0], np.float64)
    cap = 3 * int(np.prod([int(np.ceil(n * p / abs(spacing * (p if spacing < 0 else 1))) + 4)
                           for n, p in zip(dim, pix)])) + 64
    cpp = np.zeros(cap, np.float32)
    cdim = np.zeros(3, np.int32)
    stats = np.zeros(5 + 3 * int(levels), np.float64)
    rc = lib.refcuda_f3d_register(_f(_f3(ref)), _f(_f3(flo)), _i(_i3(dim)), _f(_f3(pix)), _f(_m(xyz)), _d(params),
                                  _i(cdim), _f(cpp), ctypes.c_size_t(cap), _d(stats))
    if rc != 0:
        raise RuntimeError("refcuda_f3d_register failed")
    return cpp[:3 * int(np.prod(cdim))].copy(), cdim, stats


# ----------------------------------------------------------------------------------------------
# the reference library (oracle/_ref)
# ----------------------------------------------------------------------------------------------
class Ref:
    """ctypes view of oracle/_ref/libnrref.so (the reference CPU implementation), or of
    oracle/_ref64/libnrref64.so (``Ref(REF64_SO)``: its build without the SSE path)."""

    def __init__(self, path: str = REF_SO):
        self.lib = ctypes.CDLL(path)
        self.lib.ref_nmi_value.restype = ctypes.c_double
        self.lib.ref_be_value.restype = ctypes.c_double

    def set_threads(self, n: int) -> int:
        return self.lib.ref_set_threads(int(n))

    def evaluate(self, ref, rdim, rpix, rxyz, flo, fdim, fpix, fxyz, cpp, cdim, cpix, cxyz, bins,
                 sim_weight, be_weight, pad=np.nan, fp64=False, want_def=False, want_warped=False):
        """One F3D objective-and-gradient evaluation through the reference's own functions
        (ref_evaluate.cpp): FLOAT32 images, or FLOAT64 ones with fp64=True (the FP64 oracle; only
        the ref64 build runs it through double arithmetic everywhere). Returns a dict with
        nmi, be, objective, entropies (H_ref, H_war, H_joint, total), node (3C, float64) and
        optionally def (3N) and warped (N), all float64 arrays."""
        nv, nc = int(np.prod(rdim)), int(np.prod(cdim))
        node = np.zeros(3 * nc, np.float64)
        vals = np.zeros(7, np.float64)
        d = np.zeros(3 * nv, np.float64) if want_def else None
        w = np.zeros(nv, np.float64) if want_warped else None
        fn = self.lib.ref64_evaluate if fp64 else self.lib.ref32_evaluate
        rc = fn(_f(_f3(ref)), _i(_i3(rdim)), _f(_f3(rpix)), _f(_m(rxyz)), _f(_f3(flo)), _i(_i3(fdim)),
                _f(_f3(fpix)), _f(_m(fxyz)), _f(_f3(cpp)), _i(_i3(cdim)), _f(_f3(cpix)), _f(_m(cxyz)),
                int(bins), int(bins), ctypes.c_double(sim_weight), ctypes.c_double(be_weight),
                ctypes.c_float(pad), _d(d), _d(w), _d(node), _d(vals))
        if rc != 0:
            raise RuntimeError("reference evaluation failed")
        out = dict(nmi=vals[0], be=vals[1], objective=vals[2], entropies=vals[3:7].copy(), node=node)
        if want_def:
            out["def"] = d
        if want_warped:
            out["warped"] = w
        return out

    def create_control_point_grid(self, rdim, rpix, rxyz, spacing):
        cdim = np.zeros(3, np.int32)
        cpix = np.zeros(3, np.float32)
        cxyz = np.zeros(16, np.float32)
        self.lib.ref_create_control_point_grid(_i(_i3(rdim)), _f(_f3(rpix)), _f(_m(rxyz)),
                                               _f(_f3(spacing)), _i(cdim), _f(cpix), _f(cxyz),
                                               None, ctypes.c_size_t(0))
        cpp = np.zeros(3 * int(np.prod(cdim)), np.float32)
        self.lib.ref_create_control_point_grid(_i(_i3(rdim)), _f(_f3(rpix)), _f(_m(rxyz)),
                                               _f(_f3(spacing)), _i(cdim), _f(cpix), _f(cxyz),
                                               _f(cpp), ctypes.c_size_t(cpp.size))
        return cpp, cdim, cpix, cxyz.reshape(4, 4)

    def deformation_field(self, cpp, cdim, cpix, cxyz, rdim, rpix, rxyz, mask=None):
        out = np.zeros(3 * int(np.prod(rdim)), np.float32)
        self.lib.ref_deformation_field(_f(_f3(cpp)), _i(_i3(cdim)), _f(_f3(cpix)), _f(_m(cxyz)),
                                       _i(_i3(rdim)), _f(_f3(rpix)), _f(_m(rxyz)),
                                       _i(_i3(mask)) if mask is not None else None, _f(out))
        return out

    def resample(self, flo, fdim, fpix, fxyz, dfield, rdim, rpix, rxyz, mask=None, pad=np.nan,
                 warped_init=None):
        w = np.zeros(int(np.prod(rdim)), np.float32) if warped_init is None else _f3(warped_init).copy()
        self.lib.ref_resample(_f(_f3(flo)), _i(_i3(fdim)), _f(_f3(fpix)), _f(_m(fxyz)),
                              _f(_f3(dfield)), _i(_i3(rdim)), _f(_f3(rpix)), _f(_m(rxyz)),
                              _i(_i3(mask)) if mask is not None else None, ctypes.c_float(pad), _f(w))
        return w

    def image_read(self, path):
        """(dim, nvol, pixdim, xyz, data) of a single-file NIfTI image as the reference reads it."""
        dim, nvol, pix, xyz = np.zeros(3, np.int32), ctypes.c_int(0), np.zeros(3, np.float32), np.zeros(16, np.float32)
        p = str(path).encode()
        if self.lib.ref_image_read(p, _i(dim), ctypes.byref(nvol), _f(pix), _f(xyz), None) != 0:
            raise OSError(f"reference reader failed on {path}")
        data = np.zeros(int(np.prod(dim)) * nvol.value, np.float32)
        self.lib.ref_image_read(p, _i(dim), ctypes.byref(nvol), _f(pix), _f(xyz), _f(data))
        return dim, nvol.value, pix, xyz.reshape(4, 4), data

    def resample_order(self, flo, fdim, fpix, fxyz, dfield, rdim, rpix, rxyz, order, mask=None, pad=np.nan,
                       warped_init=None):
        w = np.zeros(int(np.prod(rdim)), np.float32) if warped_init is None else _f3(warped_init).copy()
        self.lib.ref_resample_order(_f(_f3(flo)), _i(_i3(fdim)), _f(_f3(fpix)), _f(_m(fxyz)),
                                    _f(_f3(dfield)), _i(_i3(rdim)), _f(_f3(rpix)), _f(_m(rxyz)),
                                    _i(_i3(mask)) if mask is not None else None, ctypes.c_float(pad),
                                    int(order), _f(w))
        return w

    def image_gradient(self, flo, fdim, fpix, fxyz, dfield, rdim, rpix, rxyz, mask=None, pad=np.nan):
        g = np.zeros(3 * int(np.prod(rdim)), np.float32)
        self.lib.ref_image_gradient(_f(_f3(flo)), _i(_i3(fdim)), _f(_f3(fpix)), _f(_m(fxyz)),
                                    _f(_f3(dfield)), _i(_i3(rdim)), _f(_f3(rpix)), _f(_m(rxyz)),
                                    _i(_i3(mask)) if mask is not None else None,
                                    ctypes.c_float(pad), _f(g))
        return g

    def intensity_rescale(self, img, dim, new_min, new_max):
        x = _f3(img).copy()
        self.lib.ref_intensity_rescale(_f(x), _i(_i3(dim)), ctypes.c_float(new_min), ctypes.c_float(new_max))
        return x

    def nmi_value(self, ref, war, dim, ref_bins, flo_bins, mask=None, approx=True):
        total = ref_bins * flo_bins + ref_bins + flo_bins
        pro = np.zeros(total, np.float64)
        log = np.zeros(total, np.float64)
        ent = np.zeros(4, np.float64)
        v = self.lib.ref_nmi_value(_f(_f3(ref)), _f(_f3(war)), _i(_i3(dim)),
                                   _i(_i3(mask)) if mask is not None else None,
                                   int(ref_bins), int(flo_bins), int(bool(approx)),
                                   _d(pro), _d(log), _d(ent))
        return v, pro, log, ent

    def nmi_voxel_gradient(self, ref, war, war_grad, dim, ref_bins, flo_bins, weight=1.0,
                           mask=None, vgrad_init=None):
        n = int(np.prod(dim))
        vg = np.zeros(3 * n, np.float32) if vgrad_init is None else _f3(vgrad_init).copy()
        self.lib.ref_nmi_voxel_gradient(_f(_f3(ref)), _f(_f3(war)), _f(_f3(war_grad)), _i(_i3(dim)),
                                        _i(_i3(mask)) if mask is not None else None,
                                        int(ref_bins), int(flo_bins), ctypes.c_double(weight), _f(vg))
        return vg

    def convolve_to_nodes(self, vgrad, rdim, rpix, rxyz, fdim, fpix, fxyz, cdim, cpix, cxyz, weight):
        vg = _f3(vgrad).copy()
        node = np.zeros(3 * int(np.prod(cdim)), np.float32)
        self.lib.ref_convolve_to_nodes(_f(vg), _i(_i3(rdim)), _f(_f3(rpix)), _f(_m(rxyz)),
                                       _i(_i3(fdim)), _f(_f3(fpix)), _f(_m(fxyz)),
                                       _i(_i3(cdim)), _f(_f3(cpix)), _f(_m(cxyz)),
                                       ctypes.c_float(weight), _f(node))
        return vg, node

    def kernel_convolution_cubic(self, img, nvol, dim, pix, spacing, axis):
        x = _f3(img).copy()
        self.lib.ref_kernel_convolution_cubic(_f(x), int(nvol), _i(_i3(dim)), _f(_f3(pix)),
                                              ctypes.c_float(spacing), int(axis))
        return x

    def be_value(self, cpp, cdim, cpix, cxyz):
        return self.lib.ref_be_value(_f(_f3(cpp)), _i(_i3(cdim)), _f(_f3(cpix)), _f(_m(cxyz)))

    def be_gradient(self, cpp, cdim, cpix, cxyz, weight, grad_init=None):
        g = np.zeros(3 * int(np.prod(cdim)), np.float32) if grad_init is None else _f3(grad_init).copy()
        self.lib.ref_be_gradient(_f(_f3(cpp)), _i(_i3(cdim)), _f(_f3(cpix)), _f(_m(cxyz)),
                                 ctypes.c_float(weight), _f(g))
        return g

    def image_pyramid(self, img, dim, pix, xyz, levels):
        """reg_createImagePyramid<float>: list of (data [nz, ny, nx], dim, sform 4x4), coarsest first."""
        self.lib.ref_image_pyramid.restype = ctypes.c_longlong
        dims = np.zeros(3 * levels, np.int32)
        mats = np.zeros(16 * levels, np.float32)
        total = self.lib.ref_image_pyramid(_f(_f3(img)), _i(_i3(dim)), _f(_f3(pix)), _f(_m(xyz)), int(levels), None,
                                           ctypes.c_size_t(0), _i(dims), _f(mats))
        out = np.zeros(int(total), np.float32)
        self.lib.ref_image_pyramid(_f(_f3(img)), _i(_i3(dim)), _f(_f3(pix)), _f(_m(xyz)), int(levels), _f(out),
                                   ctypes.c_size_t(out.size), _i(dims), _f(mats))
        res, off = [], 0
        for l in range(levels):
            d = dims[3 * l: 3 * l + 3]
            n = int(np.prod(d))
            res.append((out[off:off + n].reshape(d[2], d[1], d[0]), tuple(int(v) for v in d),
                        mats[16 * l: 16 * l + 16].reshape(4, 4)))
            off += n
        return res

    def refine_grid(self, cpp, cdim, cpix, cxyz, rdim, rpix, rxyz):
        cap = 3 * int(np.prod([(int(c) - 3) * 2 + 8 for c in cdim]))
        out = np.zeros(cap, np.float32)
        cdo = np.zeros(3, np.int32)
        cpo = np.zeros(3, np.float32)
        cxo = np.zeros(16, np.float32)
        rc = self.lib.ref_refine_grid(_f(_f3(cpp)), _i(_i3(cdim)), _f(_f3(cpix)), _f(_m(cxyz)),
                                      _i(_i3(rdim)), _f(_f3(rpix)), _f(_m(rxyz)),
                                      _i(cdo), _f(cpo), _f(cxo), _f(out), ctypes.c_size_t(cap))
        if rc != 0:
            raise RuntimeError("ref_refine_grid: capacity")
        return out[:3 * int(np.prod(cdo))].copy(), cdo, cpo, cxo.reshape(4, 4)

    # ---- F3D2 (reg_f3d2): velocity fields --------------------------------------------------
    def velocity_def_field(self, vel, gdim, gpix, gxyz, steps, update, fdim, fpix, fxyz):
        """reg_spline_getDefFieldFromVelocityGrid: (deformation field, squaring number)."""
        out = np.zeros(3 * int(np.prod(fdim)), np.float32)
        n = ctypes.c_int(0)
        self.lib.ref_velocity_def_field(_f(_f3(vel)), _i(_i3(gdim)), _f(_f3(gpix)), _f(_m(gxyz)), int(steps),
                                        int(bool(update)), _i(_i3(fdim)), _f(_f3(fpix)), _f(_m(fxyz)), _f(out),
                                        ctypes.byref(n))
        return out, n.value

    def def_compose(self, dim, pix, xyz, apply, update):
        """reg_defField_compose: update(x) <- apply(update(x))."""
        u = _f3(update).copy()
        self.lib.ref_def_compose(_i(_i3(dim)), _f(_f3(pix)), _f(_m(xyz)), _f(_f3(apply)), _f(u))
        return u

    def exponentiate_gradient(self, fdim, fpix, fxyz, vel, gdim, gpix, gxyz, steps, vgrad):
        """Compute::ExponentiateGradient with the reference's functions."""
        g = _f3(vgrad).copy()
        self.lib.ref_exponentiate_gradient(_i(_i3(fdim)), _f(_f3(fpix)), _f(_m(fxyz)), _f(_f3(vel)), _i(_i3(gdim)),
                                           _f(_f3(gpix)), _f(_m(gxyz)), int(steps), _f(g))
        return g

    def symmetrise(self, gdim, gpix, fw_xyz, bw_xyz, fw, bw):
        """Compute::SymmetriseVelocityFields."""
        a, b = _f3(fw).copy(), _f3(bw).copy()
        self.lib.ref_symmetrise(_i(_i3(gdim)), _f(_f3(gpix)), _f(_m(fw_xyz)), _f(_m(bw_xyz)), _f(a), _f(b))
        return a, b

    def symmetric_grids(self, rdim, rpix, rxyz, fdim, fpix, fxyz, spacing):
        """reg_createSymmetricControlPointGrids: (dims, voxel->mm 4x4, identity positions)."""
        gdim, gxyz = np.zeros(3, np.int32), np.zeros(16, np.float32)
        self.lib.ref_symmetric_grids(_i(_i3(rdim)), _f(_f3(rpix)), _f(_m(rxyz)), _i(_i3(fdim)), _f(_f3(fpix)),
                                     _f(_m(fxyz)), _f(_f3(spacing)), _i(gdim), _f(gxyz), None, ctypes.c_size_t(0))
        cap = 3 * int(np.prod(gdim))
        cpp = np.zeros(cap, np.float32)
        self.lib.ref_symmetric_grids(_i(_i3(rdim)), _f(_f3(rpix)), _f(_m(rxyz)), _i(_i3(fdim)), _f(_f3(fpix)),
                                     _f(_m(fxyz)), _f(_f3(spacing)), _i(gdim), _f(gxyz), _f(cpp),
                                     ctypes.c_size_t(cap))
        return gdim, gxyz.reshape(4, 4), cpp

    def f3d2_register(self, ref, rdim, rpix, rxyz, flo, fdim, fpix, fxyz, levels, maxit, be, le, bins, spacing):
        """reg_f3d2<float>: (fw grid, bw grid, cdim, grid voxel->mm, squaring number,
        [final symmetric NMI, final weighted BE, objective calls, gradient calls])."""
        params = np.array([levels, maxit, be, le, bins, spacing, 0], np.float64)
        ext = [n * p for n, p in zip(rdim, rpix)] + [n * p for n, p in zip(fdim, fpix)]
        s = abs(spacing) * (min(list(rpix) + list(fpix)) if spacing < 0 else 1)
        cap = 3 * int(np.prod([np.ceil(2 * max(ext) / s) + 8] * 3)) + 64
        fw, bw = np.zeros(cap, np.float32), np.zeros(cap, np.float32)
        cdim, cxyz, stats = np.zeros(3, np.int32), np.zeros(16, np.float32), np.zeros(4)
        steps = ctypes.c_int(0)
        rc = self.lib.ref_f3d2_register(_f(_f3(ref)), _i(_i3(rdim)), _f(_f3(rpix)), _f(_m(rxyz)), _f(_f3(flo)),
                                        _i(_i3(fdim)), _f(_f3(fpix)), _f(_m(fxyz)), _d(params), _i(cdim), _f(fw),
                                        _f(bw), ctypes.c_size_t(cap), _f(cxyz), ctypes.byref(steps), _d(stats))
        if rc != 0:
            raise RuntimeError("ref_f3d2_register failed")
        n = 3 * int(np.prod(cdim))
        return fw[:n].copy(), bw[:n].copy(), cdim, cxyz.reshape(4, 4), steps.value, stats

    def f3d_register2(self, ref, rdim, rpix, rxyz, flo, fdim, fpix, fxyz, levels, maxit, be, le, bins, spacing):
        """reg_f3d<float> on a reference and a floating image with their own geometry: (cpp, cdim,
        grid voxel->mm, [final NMI, final weighted BE, objective calls, gradient calls])."""
        params = np.array([levels, maxit, be, le, bins, spacing, 0], np.float64)
        cap = 3 * int(np.prod([int(np.ceil(n * p / abs(spacing * (p if spacing < 0 else 1))) + 4)
                               for n, p in zip(rdim, rpix)])) + 64
        cpp, cdim, cxyz, stats = np.zeros(cap, np.float32), np.zeros(3, np.int32), np.zeros(16, np.float32), np.zeros(4)
        rc = self.lib.ref_f3d_register2(_f(_f3(ref)), _i(_i3(rdim)), _f(_f3(rpix)), _f(_m(rxyz)), _f(_f3(flo)),
                                        _i(_i3(fdim)), _f(_f3(fpix)), _f(_m(fxyz)), _d(params), _i(cdim), _f(cpp),
                                        ctypes.c_size_t(cap), _f(cxyz), _d(stats))
        if rc != 0:
            raise RuntimeError("ref_f3d_register2 failed")
        return cpp[:3 * int(np.prod(cdim))].copy(), cdim, cxyz.reshape(4, 4), stats

    def f3d_register(self, ref, flo, dim, pix, xyz, levels, maxit, be, le, bins, spacing,
                     verbose=False):
        params = np.array([levels, maxit, be, le, bins, spacing, 1 if verbose else 0], np.float64)
        cap = 3 * int(np.prod([int(np.ceil(n * p / abs(spacing * (p if spacing < 0 else 1))) + 4)
                               for n, p in zip(dim, pix)])) + 64
        cpp = np.zeros(cap, np.float32)
        cdim = np.zeros(3, np.int32)
        stats = np.zeros(5 + 3 * int(levels), np.float64)
        rc = self.lib.ref_f3d_register(_f(_f3(ref)), _f(_f3(flo)), _i(_i3(dim)), _f(_f3(pix)),
                                       _f(_m(xyz)), _d(params), _i(cdim), _f(cpp),
                                       ctypes.c_size_t(cap), _d(stats))
        if rc != 0:
            raise RuntimeError("ref_f3d_register failed")
        return cpp[:3 * int(np.prod(cdim))].copy(), cdim, stats


# ----------------------------------------------------------------------------------------------
# the C restatement (oracle/liboracle.so)
# ----------------------------------------------------------------------------------------------
class Restated:
    """ctypes view of oracle/liboracle.so (the plain-C restatement)."""

    def __init__(self, path: str = RESTATED_SO):
        build_restated()
        self.lib = ctypes.CDLL(path)
        for name in ("orc_nmi_value", "orc_be_value", "orc_max_length"):
            getattr(self.lib, name).restype = ctypes.c_double

    # ---- F3D2 (reg_f3d2): velocity fields ----------------------------------------------------
    def velocity_def_field(self, vel, gdim, gxyz, steps, update, fdim, fxyz):
        out = np.zeros(3 * int(np.prod(fdim)), np.float32)
        n = ctypes.c_int(0)
        rc = self.lib.orc_velocity_def_field(_f(_f3(vel)), _i(_i3(gdim)), _f(_m(gxyz)), int(steps), int(bool(update)),
                                             _i(_i3(fdim)), _f(_m(fxyz)), _f(out), ctypes.byref(n))
        if rc != 0:
            raise MemoryError("orc_velocity_def_field")
        return out, n.value

    def def_compose(self, dim, xyz, apply, update):
        u = _f3(update).copy()
        self.lib.orc_def_compose(_i(_i3(dim)), _f(_m(xyz)), _f(_f3(apply)), _f(u))
        return u

    def exponentiate_gradient(self, fdim, fxyz, vel, gdim, gxyz, steps, vgrad):
        g = _f3(vgrad).copy()
        rc = self.lib.orc_exponentiate_gradient(_i(_i3(fdim)), _f(_m(fxyz)), _f(_f3(vel)), _i(_i3(gdim)),
                                                _f(_m(gxyz)), int(steps), _f(g))
        if rc != 0:
            raise MemoryError("orc_exponentiate_gradient")
        return g

    def symmetrise(self, gdim, fw_xyz, bw_xyz, fw, bw):
        a, b = _f3(fw).copy(), _f3(bw).copy()
        self.lib.orc_symmetrise(_i(_i3(gdim)), _f(_m(fw_xyz)), _f(_m(bw_xyz)), _f(a), _f(b))
        return a, b

    def deformation_field(self, cpp, cdim, cpix, rdim, rpix, mask=None):
        out = np.zeros(3 * int(np.prod(rdim)), np.float32)
        rc = self.lib.orc_deformation_field(_f(_f3(cpp)), _i(_i3(cdim)), _f(_f3(cpix)), _i(_i3(rdim)),
                                            _f(_f3(rpix)), _i(_i3(mask)) if mask is not None else None,
                                            _f(out))
        if rc != 0:
            raise ValueError("control-point grid does not cover the reference image")
        return out

    def resample(self, flo, fdim, flo_ijk, dfield, rdim, mask=None, pad=np.nan, warped_init=None):
        w = np.zeros(int(np.prod(rdim)), np.float32) if warped_init is None else _f3(warped_init).copy()
        self.lib.orc_resample_linear(_f(_f3(flo)), _i(_i3(fdim)), _f(_m(flo_ijk)), _f(_f3(dfield)),
                                     _i(_i3(rdim)), _i(_i3(mask)) if mask is not None else None,
                                     ctypes.c_float(pad), _f(w))
        return w

    def resample_order(self, flo, fdim, flo_ijk, dfield, rdim, order, mask=None, pad=np.nan, warped_init=None):
        w = np.zeros(int(np.prod(rdim)), np.float32) if warped_init is None else _f3(warped_init).copy()
        rc = self.lib.orc_resample_order(_f(_f3(flo)), _i(_i3(fdim)), _f(_m(flo_ijk)), _f(_f3(dfield)),
                                         _i(_i3(rdim)), _i(_i3(mask)) if mask is not None else None,
                                         ctypes.c_float(pad), int(order), _f(w))
        if rc != 0:
            raise ValueError("orc_resample_order: order must be 0, 1 or 3")
        return w

    def image_gradient(self, flo, fdim, flo_ijk, dfield, rdim, mask=None, pad=np.nan):
        g = np.zeros(3 * int(np.prod(rdim)), np.float32)
        self.lib.orc_image_gradient_linear(_f(_f3(flo)), _i(_i3(fdim)), _f(_m(flo_ijk)),
                                           _f(_f3(dfield)), _i(_i3(rdim)),
                                           _i(_i3(mask)) if mask is not None else None,
                                           ctypes.c_float(pad), _f(g))
        return g

    def intensity_rescale(self, img, new_min, new_max):
        x = _f3(img).copy()
        self.lib.orc_intensity_rescale(_f(x), ctypes.c_size_t(x.size), ctypes.c_float(new_min),
                                       ctypes.c_float(new_max))
        return x

    def nmi_value(self, ref, war, ref_bins, flo_bins, mask=None):
        total = ref_bins * flo_bins + ref_bins + flo_bins
        pro = np.zeros(total, np.float64)
        log = np.zeros(total, np.float64)
        ent = np.zeros(4, np.float64)
        r = _f3(ref)
        v = self.lib.orc_nmi_value(_f(r), _f(_f3(war)), ctypes.c_size_t(r.size),
                                   _i(_i3(mask)) if mask is not None else None, int(ref_bins),
                                   int(flo_bins), _d(pro), _d(log), _d(ent))
        return v, pro, log, ent

    def nmi_voxel_gradient(self, ref, war, war_grad, ref_bins, flo_bins, logh, ent, weight=1.0,
                           mask=None, vgrad_init=None):
        r = _f3(ref)
        vg = np.zeros(3 * r.size, np.float32) if vgrad_init is None else _f3(vgrad_init).copy()
        self.lib.orc_nmi_voxel_gradient(_f(r), _f(_f3(war)), _f(_f3(war_grad)), ctypes.c_size_t(r.size),
                                        _i(_i3(mask)) if mask is not None else None, int(ref_bins),
                                        int(flo_bins), _d(np.ascontiguousarray(logh, np.float64)),
                                        _d(np.ascontiguousarray(ent, np.float64)),
                                        ctypes.c_double(weight), _f(vg))
        return vg

    def kernel_convolution_cubic(self, img, nvol, dim, pix, spacing, axis, mask=None):
        x = _f3(img).copy()
        self.lib.orc_kernel_convolution_cubic(_f(x), int(nvol), _i(_i3(dim)), _f(_f3(pix)),
                                              ctypes.c_float(spacing), int(axis),
                                              _i(_i3(mask)) if mask is not None else None)
        return x

    def convolve_to_nodes(self, vgrad, rdim, rpix, ref_ijk, cdim, cpix, grid_xyz, flo_ijk, weight):
        vg = _f3(vgrad).copy()
        node = np.zeros(3 * int(np.prod(cdim)), np.float32)
        self.lib.orc_convolve_to_nodes(_f(vg), _i(_i3(rdim)), _f(_f3(rpix)), _f(_m(ref_ijk)),
                                       _i(_i3(cdim)), _f(_f3(cpix)), _f(_m(grid_xyz)),
                                       _f(_m(flo_ijk)), ctypes.c_float(weight), _f(node))
        return vg, node

    def voxel_to_node(self, voxel, rdim, rpix, ref_ijk, cdim, grid_xyz, reorient, weight):
        node = np.zeros(3 * int(np.prod(cdim)), np.float32)
        self.lib.orc_voxel_to_node(_f(node), _i(_i3(cdim)), _f(_m(grid_xyz)), _f(_f3(voxel)),
                                   _i(_i3(rdim)), _f(_f3(rpix)), _f(_m(ref_ijk)), _f(_m(reorient)),
                                   ctypes.c_float(weight), 0)
        return node

    def be_value(self, cpp, cdim):
        return self.lib.orc_be_value(_f(_f3(cpp)), _i(_i3(cdim)))

    def be_gradient(self, cpp, cdim, grid_xyz, weight, grad_init=None):
        g = np.zeros(3 * int(np.prod(cdim)), np.float32) if grad_init is None else _f3(grad_init).copy()
        self.lib.orc_be_gradient(_f(_f3(cpp)), _i(_i3(cdim)), _f(_m(grid_xyz)), ctypes.c_float(weight), _f(g))
        return g

    def max_length(self, grad, nnode):
        return self.lib.orc_max_length(_f(_f3(grad)), ctypes.c_size_t(nnode), 1, 1, 1)

    def normalise_gradient(self, grad, nnode, maxlen):
        g = _f3(grad).copy()
        self.lib.orc_normalise_gradient(_f(g), ctypes.c_size_t(nnode), ctypes.c_double(maxlen), 1, 1, 1)
        return g

    def update_control_points(self, best, grad, scale):
        cur = np.zeros_like(_f3(best))
        self.lib.orc_update_control_points(_f(cur), _f(_f3(best)), _f(_f3(grad)), ctypes.c_float(scale),
                                           ctypes.c_size_t(cur.size))
        return cur

    def cg_update(self, grad, g1, g2, first_call):
        grad, g1, g2 = _f3(grad).copy(), _f3(g1).copy(), _f3(g2).copy()
        self.lib.orc_cg_update(_f(grad), _f(g1), _f(g2), ctypes.c_size_t(grad.size), int(bool(first_call)))
        return grad, g1, g2
