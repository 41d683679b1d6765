"""niftyreg_b200 -- B200-native F3D objective-and-gradient evaluation (NiftyReg reg_f3d path).

The product is the shared library ``libniftyreg_b200.so`` (CUDA kernels for sm_100a, the C ABI
declared in ``include/niftyreg_b200.h`` and the registration driver). This module is a thin
ctypes binding to that ABI: array arguments are device pointers (``int`` addresses, e.g.
``tensor.data_ptr()``) unless a function says it takes host arrays. There is no fallback: if the
library is missing or no sm_100 device is present, calls raise.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libniftyreg_b200.so")

__all__ = [
    "NrbError", "Geometry", "Objective", "F3dParams", "F3dResult", "lib", "build",
    "make_geometry", "identity_header", "Nmi", "Workspace",
]


class NrbError(RuntimeError):
    """A C-ABI call returned a non-zero nrb_status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"nrb_status {status}: {message}")
        self.status = status


_M16 = ctypes.c_float * 16
_I3 = ctypes.c_int32 * 3
_F3 = ctypes.c_float * 3


class Geometry(ctypes.Structure):
    _fields_ = [
        ("ref_dim", _I3), ("ref_pixdim", _F3), ("ref_xyz", _M16), ("ref_ijk", _M16),
        ("flo_dim", _I3), ("flo_pixdim", _F3), ("flo_xyz", _M16), ("flo_ijk", _M16),
        ("cpp_dim", _I3), ("cpp_pixdim", _F3), ("cpp_xyz", _M16), ("cpp_ijk", _M16),
    ]

    @property
    def ref_nvox(self) -> int:
        return int(np.prod(list(self.ref_dim)))

    @property
    def cpp_nvox(self) -> int:
        return int(np.prod(list(self.cpp_dim)))


class Objective(ctypes.Structure):
    _fields_ = [("nmi", ctypes.c_double), ("entropy", ctypes.c_double * 4), ("be", ctypes.c_double),
                ("objective", ctypes.c_double), ("max_grad_len", ctypes.c_double)]


class F3dParams(ctypes.Structure):
    _fields_ = [("levels", ctypes.c_int32), ("max_iterations", ctypes.c_int32),
                ("bending_energy", ctypes.c_float), ("spacing", _F3), ("ref_bins", ctypes.c_int32),
                ("flo_bins", ctypes.c_int32), ("padding", ctypes.c_float), ("verbose", ctypes.c_int32),
                ("host_loop", ctypes.c_int32), ("floating_margin", ctypes.c_int32),
                ("batch_gradient_percent", ctypes.c_int32), ("floating_texture", ctypes.c_int32),
                ("autotune", ctypes.c_int32), ("batch_group_mb", ctypes.c_int32)]


class WalkEntry(ctypes.Structure):
    """nrb_walk_entry: one shape of the walk autotuner's table."""
    _fields_ = [("ref_dim", _I3), ("cpp_dim", _I3), ("bins", ctypes.c_int32 * 2), ("obj_ty", ctypes.c_int32),
                ("obj_zchunk", ctypes.c_int32), ("obj_resident", ctypes.c_int32), ("obj_us", ctypes.c_float),
                ("obj_model_us", ctypes.c_float), ("grad_ty", ctypes.c_int32), ("grad_zchunk", ctypes.c_int32),
                ("grad_resident", ctypes.c_int32), ("grad_us", ctypes.c_float), ("grad_model_us", ctypes.c_float),
                ("candidates", ctypes.c_int32)]


class Image(ctypes.Structure):
    """nrb_image: a host NIfTI image (float32 data, orientation as NiftyReg picks it)."""
    _fields_ = [("dim", _I3), ("nvol", ctypes.c_int32), ("pixdim", _F3), ("xyz", ctypes.c_float * 16),
                ("ijk", ctypes.c_float * 16), ("sform_code", ctypes.c_int32), ("qform_code", ctypes.c_int32),
                ("intent_code", ctypes.c_int32),
                ("intent_p1", ctypes.c_float), ("intent_p2", ctypes.c_float), ("intent_name", ctypes.c_char * 16),
                ("data", ctypes.POINTER(ctypes.c_float))]


class F3dResult(ctypes.Structure):
    _fields_ = [("cpp_dim", _I3), ("final_nmi", ctypes.c_double), ("final_be", ctypes.c_double),
                ("final_objective", ctypes.c_double), ("objective_evaluations", ctypes.c_int64),
                ("gradient_evaluations", ctypes.c_int64), ("seconds", ctypes.c_double)]


_LIB = None


def build(force: bool = False) -> str:
    """Compiles libniftyreg_b200.so for sm_100a with nvcc (no GPU needed)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.check_call(["make", "-C", HERE, "-j4"], stdout=subprocess.DEVNULL)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    """The loaded C ABI. Raises if the shared library has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run niftyreg_b200.build() (nvcc, sm_100a)")
        L = ctypes.CDLL(LIB_PATH)
        L.nrb_last_error.restype = ctypes.c_char_p
        L.nrb_kernel_launch_count.restype = ctypes.c_int64
        L.nrb_nmi_destroy.restype = None
        L.nrb_workspace_destroy.restype = None
        L.nrb_f3d_default_params.restype = None
        _LIB = L
    return _LIB


def check(status: int):
    if status != 0:
        raise NrbError(status, lib().nrb_last_error().decode())


def _p(x):
    """Device pointer argument: an int address, an object with data_ptr(), or None."""
    if x is None:
        return None
    if hasattr(x, "data_ptr"):
        return ctypes.c_void_p(x.data_ptr())
    return ctypes.c_void_p(int(x))


def _s(stream):
    if stream is None:
        return None
    if hasattr(stream, "cuda_stream"):
        return ctypes.c_void_p(stream.cuda_stream)
    return ctypes.c_void_p(int(stream))


def _inv(m):
    return np.linalg.inv(np.asarray(m, np.float64).reshape(4, 4)).astype(np.float32)


def identity_header(pixdim, origin=(0.0, 0.0, 0.0)):
    """voxel->mm matrix of an image with identity orientation."""
    m = np.eye(4, dtype=np.float32)
    for i in range(3):
        m[i, i] = pixdim[i]
        m[i, 3] = origin[i]
    return m


def make_geometry(ref_dim, ref_pixdim, ref_xyz, flo_dim, flo_pixdim, flo_xyz, cpp_dim, cpp_pixdim,
                  cpp_xyz) -> Geometry:
    g = Geometry()
    for name, dim, pix, xyz in (("ref", ref_dim, ref_pixdim, ref_xyz), ("flo", flo_dim, flo_pixdim, flo_xyz),
                                ("cpp", cpp_dim, cpp_pixdim, cpp_xyz)):
        getattr(g, name + "_dim")[:] = [int(v) for v in dim]
        getattr(g, name + "_pixdim")[:] = [float(v) for v in pix]
        getattr(g, name + "_xyz")[:] = [float(v) for v in np.asarray(xyz, np.float32).reshape(16)]
        getattr(g, name + "_ijk")[:] = [float(v) for v in _inv(xyz).reshape(16)]
    return g


def control_grid_header(ref_dim, ref_pixdim, spacing_mm):
    """Dims, spacing and voxel->mm of reg_createControlPointGrid for an identity-oriented
    reference (node 0 one spacing before voxel 0)."""
    dim = []
    for n, d, s in zip(ref_dim, ref_pixdim, spacing_mm):
        v = np.float32(np.float32(n) * np.float32(d) / np.float32(s) + np.float32(3.0))
        i = int(v)
        dim.append(i + (1 if v > i else 0))
    xyz = identity_header(spacing_mm, [-float(s) for s in spacing_mm])
    return dim, [float(s) for s in spacing_mm], xyz


class Nmi:
    """NMI measure workspace (joint histogram, FP64 tables) on the current device."""

    def __init__(self, ref_bins: int, flo_bins: int):
        self.h = ctypes.c_void_p()
        self.ref_bins, self.flo_bins = ref_bins, flo_bins
        check(lib().nrb_nmi_create(int(ref_bins), int(flo_bins), ctypes.byref(self.h)))

    def close(self):
        if self.h:
            lib().nrb_nmi_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tables(self, stream=None):
        total = self.ref_bins * self.flo_bins + self.ref_bins + self.flo_bins
        pro = np.zeros(total, np.float64)
        log = np.zeros(total, np.float64)
        ent = np.zeros(4, np.float64)
        check(lib().nrb_nmi_read_tables(self.h, pro.ctypes.data_as(ctypes.c_void_p),
                                        log.ctypes.data_as(ctypes.c_void_p),
                                        ent.ctypes.data_as(ctypes.c_void_p), _s(stream)))
        return pro, log, ent


class Workspace:
    """Scratch buffers of one registration level (nrb_workspace_create)."""

    def __init__(self, g: Geometry):
        self.h = ctypes.c_void_p()
        self.g = g
        check(lib().nrb_workspace_create(ctypes.byref(g), ctypes.byref(self.h)))

    def close(self):
        if self.h:
            lib().nrb_workspace_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------------------------------------
# Compute / reg_nmi operations (device pointers)
# ------------------------------------------------------------------------------------------------
def get_deformation_field(g, cpp, deformation, mask=None, stream=None):
    check(lib().nrb_get_deformation_field(ctypes.byref(g), _p(cpp), _p(mask), _p(deformation), _s(stream)))


def resample_image(g, flo, deformation, warped, padding=math.nan, mask=None, stream=None):
    check(lib().nrb_resample_image(ctypes.byref(g), _p(flo), _p(deformation), _p(mask), ctypes.c_float(padding),
                                   _p(warped), _s(stream)))


def read_image(path):
    """A NIfTI-1 file (.nii, .nii.gz) as (data [nvol, nz, ny, nx] float32, pixdim, xyz 4x4), read as
    NiftyReg reads it."""
    img = Image()
    check(lib().nrb_image_read(str(path).encode(), ctypes.byref(img)))
    try:
        nx, ny, nz = list(img.dim)
        n = nx * ny * nz * img.nvol
        data = np.ctypeslib.as_array(img.data, shape=(n,)).copy().reshape(img.nvol, nz, ny, nx)
        return data, tuple(float(v) for v in img.pixdim), np.array(img.xyz, np.float32).reshape(4, 4)
    finally:
        lib().nrb_image_free(ctypes.byref(img))


def write_image(path, data, pixdim, xyz, intent_code=0, intent_p1=0.0, intent_name=b""):
    """Writes data [nvol, nz, ny, nx] (or [nz, ny, nx]) as a float32 NIfTI-1 file with xyz as the sform."""
    a = np.ascontiguousarray(data, np.float32)
    if a.ndim == 3:
        a = a[None]
    nvol, nz, ny, nx = a.shape
    img = Image()
    img.dim[:] = [nx, ny, nz]
    img.nvol = nvol
    img.pixdim[:] = [float(v) for v in pixdim]
    img.xyz[:] = [float(v) for v in np.asarray(xyz, np.float32).reshape(16)]
    img.sform_code = 1
    img.intent_code = int(intent_code)
    img.intent_p1 = float(intent_p1)
    img.intent_name = intent_name
    img.data = a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    check(lib().nrb_image_write(str(path).encode(), ctypes.byref(img)))


# ---- F3D2 (reg_f3d2): symmetric registration with velocity fields ----------------------------
def get_def_field_from_velocity_grid(g, vel, steps, deformation, update=False, stream=None):
    """Compute::GetDefFieldFromVelocityGrid: deformation field on g's reference grid from the
    velocity grid `vel` (g's grid); returns the squaring number used."""
    n = ctypes.c_int32(int(steps))
    check(lib().nrb_get_def_field_from_velocity_grid(ctypes.byref(g), _p(vel), int(bool(update)), ctypes.byref(n),
                                                     _p(deformation), _s(stream)))
    return n.value


def def_field_compose(dim, xyz, apply, update, stream=None):
    """reg_defField_compose: update(x) <- apply(update(x)) on a field of dims `dim`, voxel->mm `xyz`."""
    m = np.asarray(xyz, np.float32).reshape(16)
    x16, i16 = (ctypes.c_float * 16)(*[float(v) for v in m]), (ctypes.c_float * 16)(*[float(v) for v in _inv(m).ravel()])
    check(lib().nrb_def_field_compose(_I3(*[int(v) for v in dim]), x16, i16, _p(apply), _p(update), _s(stream)))


def exponentiate_gradient(g, vel_other, steps, vgrad, stream=None):
    """Compute::ExponentiateGradient: vgrad (on g's reference grid) along the velocity grid
    `vel_other` (g's grid), in place."""
    check(lib().nrb_exponentiate_gradient(ctypes.byref(g), _p(vel_other), int(steps), _p(vgrad), _s(stream)))


def symmetrise_velocity_fields(g_fw, fw, g_bw, bw, stream=None):
    """Compute::SymmetriseVelocityFields on the two grids, in place."""
    check(lib().nrb_symmetrise_velocity_fields(ctypes.byref(g_fw), _p(fw), ctypes.byref(g_bw), _p(bw), _s(stream)))


def f3d2_register_images(ref, ref_pixdim, ref_xyz, flo, flo_pixdim, flo_xyz, params, warped=True):
    """reg_f3d2 (-vel) on two host volumes ([nz, ny, nx]) with their own voxel->mm matrices.
    Returns (fw grid [3, cz, cy, cx], bw grid, grid voxel->mm 4x4 (fw, bw), squaring number,
    warped floating on the reference grid or None, warped reference on the floating grid or None,
    result)."""
    r, keep_r = _image_of(ref, ref_pixdim, ref_xyz)
    f, keep_f = _image_of(flo, flo_pixdim, flo_xyz)
    cf, cb, wf, wb, res = Image(), Image(), Image(), Image(), F3dResult()
    check(lib().nrb_f3d2_register_images(ctypes.byref(r), ctypes.byref(f), ctypes.byref(params), ctypes.byref(cf),
                                         ctypes.byref(cb), ctypes.byref(wf) if warped else None,
                                         ctypes.byref(wb) if warped else None, ctypes.byref(res)))
    try:
        def grid(img):
            cx, cy, cz = list(img.dim)
            return (np.ctypeslib.as_array(img.data, shape=(3 * cx * cy * cz,)).copy().reshape(3, cz, cy, cx),
                    np.array(img.xyz, np.float32).reshape(4, 4))

        gf, xf = grid(cf)
        gb, xb = grid(cb)
        outs = [None, None]
        if warped:
            for k, (img, like) in enumerate(((wf, ref), (wb, flo))):
                nz, ny, nx = np.shape(like)
                outs[k] = np.ctypeslib.as_array(img.data, shape=(nx * ny * nz,)).copy().reshape(nz, ny, nx)
        return gf, gb, (xf, xb), int(cf.intent_p2), outs[0], outs[1], res
    finally:
        for img in (cf, cb) + ((wf, wb) if warped else ()):
            lib().nrb_image_free(ctypes.byref(img))


def _header_image(dim, pix, xyz):
    i = Image()
    i.dim[:] = [int(v) for v in dim]
    i.nvol = 1
    i.pixdim[:] = [float(v) for v in pix]
    i.xyz[:] = [float(v) for v in np.asarray(xyz, np.float32).ravel()]
    i.sform_code = 1
    return i


def f3d_grid_header(ref_dim, ref_pixdim, ref_xyz, params):
    """(dims, spacing, voxel->mm 4x4) of the final control-point grid of a reg_f3d registration
    of a reference with this header (host only)."""
    r = _header_image(ref_dim, ref_pixdim, ref_xyz)
    d, pix, x = _I3(), (ctypes.c_float * 3)(), (ctypes.c_float * 16)()
    check(lib().nrb_f3d_grid_header(ctypes.byref(r), ctypes.byref(params), d, pix, x))
    return list(d), list(pix), np.array(list(x), np.float32).reshape(4, 4)


def f3d2_grid_header(ref_dim, ref_pixdim, ref_xyz, flo_dim, flo_pixdim, flo_xyz, params):
    """(dims, spacing, voxel->mm 4x4) of the final velocity grids of a reg_f3d2 registration of
    images with these headers (host only)."""
    def img(dim, pix, xyz):
        i = Image()
        i.dim[:] = [int(v) for v in dim]
        i.nvol = 1
        i.pixdim[:] = [float(v) for v in pix]
        i.xyz[:] = [float(v) for v in np.asarray(xyz, np.float32).ravel()]
        i.sform_code = 1
        return i
    r, f = img(ref_dim, ref_pixdim, ref_xyz), img(flo_dim, flo_pixdim, flo_xyz)
    d, pix, x = _I3(), (ctypes.c_float * 3)(), (ctypes.c_float * 16)()
    check(lib().nrb_f3d2_grid_header(ctypes.byref(r), ctypes.byref(f), ctypes.byref(params), d, pix, x))
    return list(d), list(pix), np.array(list(x), np.float32).reshape(4, 4)


def f3d2_register_files(ref_path, flo_path, params, cpp_path, res_path=None):
    """A reg_f3d -vel request on NIfTI files: the backward grid (and warped reference) are written
    beside the forward ones with "_backward" before the extension."""
    res = F3dResult()
    check(lib().nrb_f3d2_register_files(str(ref_path).encode(), str(flo_path).encode(), ctypes.byref(params),
                                        str(cpp_path).encode(), str(res_path).encode() if res_path else None,
                                        ctypes.byref(res)))
    return res


def _image_of(data, pixdim, xyz, sform_code=1):
    a = np.ascontiguousarray(data, np.float32)
    nz, ny, nx = a.shape
    img = Image()
    img.dim[:] = [nx, ny, nz]
    img.nvol = 1
    img.pixdim[:] = [float(v) for v in pixdim]
    m = np.asarray(xyz, np.float32).reshape(4, 4)
    img.xyz[:] = [float(v) for v in m.ravel()]
    img.ijk[:] = [float(v) for v in _inv(m).ravel()]
    img.sform_code = int(sform_code)
    img.data = a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    return img, a


def register_images(ref, ref_pixdim, ref_xyz, flo, flo_pixdim, flo_xyz, params, warped=True, sform_code=1):
    """reg_f3d on two host volumes ([nz, ny, nx]) with their own spacings and voxel->mm matrices.
    Returns (cpp [3, cz, cy, cx], grid voxel->mm 4x4, warped image or None, result)."""
    r, keep_r = _image_of(ref, ref_pixdim, ref_xyz, sform_code)
    f, keep_f = _image_of(flo, flo_pixdim, flo_xyz, sform_code)
    cpp, w, res = Image(), Image(), F3dResult()
    check(lib().nrb_f3d_register_images(ctypes.byref(r), ctypes.byref(f), ctypes.byref(params), ctypes.byref(cpp),
                                        ctypes.byref(w) if warped else None, ctypes.byref(res)))
    try:
        cx, cy, cz = list(cpp.dim)
        grid = np.ctypeslib.as_array(cpp.data, shape=(3 * cx * cy * cz,)).copy().reshape(3, cz, cy, cx)
        gxyz = np.array(cpp.xyz, np.float32).reshape(4, 4)
        out = None
        if warped:
            nz, ny, nx = np.shape(ref)
            out = np.ctypeslib.as_array(w.data, shape=(nx * ny * nz,)).copy().reshape(nz, ny, nx)
        return grid, gxyz, out, res
    finally:
        lib().nrb_image_free(ctypes.byref(cpp))
        if warped:
            lib().nrb_image_free(ctypes.byref(w))


def register_files(ref_path, flo_path, params, cpp_path, res_path=None):
    """A registration request on NIfTI files (reg_f3d -ref -flo -cpp [-res])."""
    res = F3dResult()
    check(lib().nrb_f3d_register_files(str(ref_path).encode(), str(flo_path).encode(), ctypes.byref(params),
                                       str(cpp_path).encode(), str(res_path).encode() if res_path else None,
                                       ctypes.byref(res)))
    return res


def resample_image_order(g, flo, deformation, warped, order, padding=math.nan, mask=None, stream=None):
    """Warp with interpolation `order` (0 nearest, 1 linear, 3 cubic spline), bit-identical to the
    reference's ResampleImage3D."""
    check(lib().nrb_resample_image_order(ctypes.byref(g), _p(flo), _p(deformation), _p(mask), int(order),
                                         ctypes.c_float(padding), _p(warped), _s(stream)))


def f3d_warped_image(g, flo, cpp, warped, order=3, padding=math.nan, stream=None):
    """reg_f3d::GetWarpedImage on the device: deformation field of `cpp` over the reference
    geometry of `g`, then the floating image resampled with `order` (cubic spline by default)."""
    check(lib().nrb_f3d_warped_image(ctypes.byref(g), _p(flo), _p(cpp), int(order), ctypes.c_float(padding),
                                     _p(warped), _s(stream)))


def image_pyramid_headers(dim, pixdim, xyz, levels):
    """(dims [levels x 3], xyz [levels x 4 x 4], total floats) of reg_createImagePyramid for an
    image of these dims, spacings and voxel -> mm matrix (host only), coarsest level first."""
    dims = np.zeros(3 * levels, np.int32)
    mats = np.zeros(16 * levels, np.float32)
    total = ctypes.c_int64()
    x16 = (ctypes.c_float * 16)(*[float(v) for v in np.asarray(xyz, np.float32).ravel()]) if xyz is not None else None
    check(lib().nrb_image_pyramid(None, _I3(*[int(v) for v in dim]), _F3(*[float(v) for v in pixdim]), x16,
                                  int(levels), None, ctypes.c_int64(0), dims.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                  mats.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ctypes.byref(total), None))
    return dims.reshape(levels, 3), mats.reshape(levels, 4, 4), total.value


def image_pyramid(img, dim, pixdim, xyz, levels, out, stream=None):
    """reg_createImagePyramid<float> on the device: `out` (device, >= total floats) receives the
    levels end to end, coarsest first. Returns the headers as image_pyramid_headers does."""
    dims, mats, total = image_pyramid_headers(dim, pixdim, xyz, levels)
    x16 = (ctypes.c_float * 16)(*[float(v) for v in np.asarray(xyz, np.float32).ravel()]) if xyz is not None else None
    check(lib().nrb_image_pyramid(_p(img), _I3(*[int(v) for v in dim]), _F3(*[float(v) for v in pixdim]), x16,
                                  int(levels), _p(out), ctypes.c_int64(total), None, None, None, _s(stream)))
    return dims, mats, total


def refine_control_point_grid(old, old_dim, out, new_dim, stream=None):
    """reg_spline_refineControlPointGrid3D's node values: `old` (old_dim nodes, three planes)
    refined onto new_dim nodes at half the spacing, into `out` (device)."""
    check(lib().nrb_refine_control_point_grid(_p(old), _I3(*[int(v) for v in old_dim]), _p(out),
                                              _I3(*[int(v) for v in new_dim]), _s(stream)))


def get_image_gradient(g, flo, deformation, grad, padding=math.nan, mask=None, stream=None):
    check(lib().nrb_get_image_gradient(ctypes.byref(g), _p(flo), _p(deformation), _p(mask), ctypes.c_float(padding),
                                       _p(grad), _s(stream)))


def intensity_rescale(img, nvox, new_min, new_max, stream=None):
    check(lib().nrb_intensity_rescale(_p(img), ctypes.c_int64(nvox), ctypes.c_float(new_min),
                                      ctypes.c_float(new_max), _s(stream)))


def nmi_value(nmi: Nmi, g, ref, warped, mask=None, obj=None, stream=None) -> float:
    out = ctypes.c_double()
    check(lib().nrb_nmi_value(nmi.h, ctypes.byref(g), _p(ref), _p(warped), _p(mask), _p(obj), ctypes.byref(out),
                              _s(stream)))
    return out.value


def nmi_voxel_gradient(nmi: Nmi, g, ref, warped, warped_grad, vgrad, weight=1.0, mask=None, stream=None):
    check(lib().nrb_nmi_voxel_gradient(nmi.h, ctypes.byref(g), _p(ref), _p(warped), _p(warped_grad), _p(mask),
                                       ctypes.c_double(weight), _p(vgrad), _s(stream)))


def kernel_convolution_cubic(img, nvol, dim, pixdim, spacing_mm, axis, stream=None):
    d = _I3(*[int(v) for v in dim])
    p = _F3(*[float(v) for v in pixdim])
    check(lib().nrb_kernel_convolution_cubic(_p(img), int(nvol), d, p, ctypes.c_float(spacing_mm), int(axis),
                                             _s(stream)))


def convolve_voxel_based_gradient(ws: Workspace, vgrad, node_grad, weight, stream=None):
    check(lib().nrb_convolve_voxel_based_gradient(ws.h, ctypes.byref(ws.g), _p(vgrad), ctypes.c_float(weight),
                                                  _p(node_grad), _s(stream)))


def approx_bending_energy(ws: Workspace, cpp, stream=None) -> float:
    out = ctypes.c_double()
    check(lib().nrb_approx_bending_energy(ws.h, ctypes.byref(ws.g), _p(cpp), None, ctypes.byref(out), _s(stream)))
    return out.value


def approx_bending_energy_gradient(ws: Workspace, cpp, node_grad, weight, stream=None):
    check(lib().nrb_approx_bending_energy_gradient(ws.h, ctypes.byref(ws.g), _p(cpp), ctypes.c_float(weight),
                                                   _p(node_grad), _s(stream)))


def get_maximal_length(node_grad, nnode, stream=None) -> float:
    out = ctypes.c_double()
    check(lib().nrb_get_maximal_length(_p(node_grad), ctypes.c_int64(nnode), None, ctypes.byref(out), _s(stream)))
    return out.value


def normalise_gradient(node_grad, nnode, max_len, stream=None):
    check(lib().nrb_normalise_gradient(_p(node_grad), ctypes.c_int64(nnode), ctypes.c_double(max_len), None,
                                       _s(stream)))


def update_control_point_position(cur, best, grad, scale, n, stream=None):
    check(lib().nrb_update_control_point_position(_p(cur), _p(best), _p(grad), ctypes.c_float(scale),
                                                  ctypes.c_int64(n), _s(stream)))


def conjugate_gradient(ws: Workspace, grad, g1, g2, n, first_call, stream=None):
    check(lib().nrb_conjugate_gradient(ws.h, _p(grad), _p(g1), _p(g2), ctypes.c_int64(n), int(bool(first_call)),
                                       _s(stream)))


def f3d_objective(ws: Workspace, nmi: Nmi, ref, flo, cpp, sim_weight, be_weight, padding=math.nan, mask=None,
                  obj=None, stream=None) -> Objective:
    out = Objective()
    check(lib().nrb_f3d_objective(ws.h, nmi.h, ctypes.byref(ws.g), _p(ref), _p(flo), _p(mask), _p(cpp),
                                  ctypes.c_float(padding), ctypes.c_double(sim_weight), ctypes.c_double(be_weight),
                                  _p(obj), ctypes.byref(out), _s(stream)))
    return out


def f3d_gradient(ws: Workspace, nmi: Nmi, ref, flo, cpp, vgrad, node_grad, sim_weight, be_weight,
                 padding=math.nan, mask=None, stream=None):
    check(lib().nrb_f3d_gradient(ws.h, nmi.h, ctypes.byref(ws.g), _p(ref), _p(flo), _p(mask), _p(cpp),
                                 ctypes.c_float(padding), ctypes.c_double(sim_weight), ctypes.c_double(be_weight),
                                 _p(vgrad), _p(node_grad), _s(stream)))


def default_params(**kw) -> F3dParams:
    p = F3dParams()
    lib().nrb_f3d_default_params(ctypes.byref(p))
    for k, v in kw.items():
        if k == "spacing":
            v = list(v) + [math.nan] * (3 - len(v))
            p.spacing[:] = [float(x) for x in v]
        else:
            setattr(p, k, v)
    return p


def grid_dims(dim, pixdim, params: F3dParams):
    out = _I3()
    check(lib().nrb_f3d_grid_dims(_I3(*[int(v) for v in dim]), _F3(*[float(v) for v in pixdim]),
                                  ctypes.byref(params), out))
    return [int(v) for v in out]


def register_host(ref: np.ndarray, flo: np.ndarray, pixdim, params: F3dParams):
    """Full F3D registration of host volumes ([nz, ny, nx] float32). Returns (cpp, result):
    cpp is [3, cz, cy, cx] float32 (control-point positions in mm)."""
    ref = np.ascontiguousarray(ref, np.float32)
    flo = np.ascontiguousarray(flo, np.float32)
    nz, ny, nx = ref.shape
    dim = _I3(nx, ny, nz)
    cd = grid_dims((nx, ny, nz), pixdim, params)
    cpp = np.zeros((3, cd[2], cd[1], cd[0]), np.float32)
    res = F3dResult()
    check(lib().nrb_f3d_register_host(ref.ctypes.data_as(ctypes.c_void_p), flo.ctypes.data_as(ctypes.c_void_p), dim,
                                      _F3(*[float(v) for v in pixdim]), ctypes.byref(params),
                                      cpp.ctypes.data_as(ctypes.c_void_p), ctypes.c_int64(cpp.size),
                                      ctypes.byref(res)))
    return cpp, res


class PairDesc(ctypes.Structure):
    """nrb_pair: one registration request with host images."""
    _fields_ = [("ref_host", ctypes.c_void_p), ("flo_host", ctypes.c_void_p), ("dim", _I3), ("pixdim", _F3),
                ("cpp_out_host", ctypes.c_void_p), ("cpp_capacity", ctypes.c_int64)]


def footprint(dim, pixdim, params: F3dParams) -> int:
    """Peak device bytes of one registration (the server's admission unit)."""
    out = ctypes.c_int64()
    check(lib().nrb_f3d_footprint(_I3(*[int(v) for v in dim]), _F3(*[float(v) for v in pixdim]),
                                  ctypes.byref(params), ctypes.byref(out)))
    return int(out.value)


class _Request:
    """Host buffers of one request, kept alive until its result is read."""

    def __init__(self, ref, flo, pixdim, params):
        self.ref = np.ascontiguousarray(ref, np.float32)
        self.flo = np.ascontiguousarray(flo, np.float32)
        nz, ny, nx = self.ref.shape
        cd = grid_dims((nx, ny, nz), pixdim, params)
        self.cpp = np.zeros((3, cd[2], cd[1], cd[0]), np.float32)
        self.params = params
        self.desc = PairDesc(self.ref.ctypes.data, self.flo.ctypes.data, _I3(nx, ny, nz),
                             _F3(*[float(v) for v in pixdim]), self.cpp.ctypes.data, self.cpp.size)


class Server:
    """Continuous-batching registration server on the current device (nrb_server_*): `slots`
    workers, each registering a group of up to `max_group` queued requests of similar size at a
    time through the batched engine, admitted in arrival order against an HBM budget in bytes
    (0 = 80% of the free device memory)."""

    def __init__(self, slots: int, budget_bytes: int = 0, max_group: int = 16):
        self.h = ctypes.c_void_p()
        L = lib()
        L.nrb_server_destroy.restype = None
        check(L.nrb_server_create_grouped(int(slots), int(max_group), ctypes.c_int64(budget_bytes),
                                          ctypes.byref(self.h)))
        self._pending = {}

    def submit(self, ref, flo, pixdim, params: F3dParams) -> int:
        req = _Request(ref, flo, pixdim, params)
        t = ctypes.c_int64()
        check(lib().nrb_server_submit(self.h, ctypes.byref(req.desc), ctypes.byref(params), ctypes.byref(t)))
        self._pending[t.value] = req
        return int(t.value)

    def wait(self, ticket: int):
        """(cpp [3, cz, cy, cx], F3dResult, queue seconds, latency seconds)."""
        res, q, lat = F3dResult(), ctypes.c_double(), ctypes.c_double()
        try:
            check(lib().nrb_server_wait(self.h, ctypes.c_int64(ticket), ctypes.byref(res), ctypes.byref(q),
                                        ctypes.byref(lat)))
        finally:
            req = self._pending.pop(ticket, None)
        return req.cpp, res, q.value, lat.value

    def stats(self):
        """(peak admitted bytes, peak concurrent registrations)."""
        b, a = ctypes.c_int64(), ctypes.c_int32()
        check(lib().nrb_server_stats(self.h, ctypes.byref(b), ctypes.byref(a)))
        return int(b.value), int(a.value)

    def peak_group(self) -> int:
        g = ctypes.c_int32()
        check(lib().nrb_server_peak_group(self.h, ctypes.byref(g)))
        return int(g.value)

    def close(self):
        if self.h:
            lib().nrb_server_destroy(self.h)
            self.h = ctypes.c_void_p()
            self._pending.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def register_batch(pairs, params: F3dParams, concurrency: int, budget_bytes: int = 0):
    """pairs: list of (ref, flo, pixdim) host volumes. Returns [(cpp, F3dResult)] in order."""
    reqs = [_Request(r, f, p, params) for r, f, p in pairs]
    descs = (PairDesc * len(reqs))(*[q.desc for q in reqs])
    results = (F3dResult * len(reqs))()
    check(lib().nrb_f3d_register_batch(descs, len(reqs), ctypes.byref(params), int(concurrency),
                                       ctypes.c_int64(budget_bytes), results))
    return [(q.cpp, results[i]) for i, q in enumerate(reqs)]


def register_device(ref, flo, dim, pixdim, params: F3dParams, cpp_out, capacity, stream=None) -> F3dResult:
    """Full F3D registration of device-resident volumes; cpp_out is a device buffer."""
    res = F3dResult()
    check(lib().nrb_f3d_register_device(_p(ref), _p(flo), _I3(*[int(v) for v in dim]),
                                        _F3(*[float(v) for v in pixdim]), ctypes.byref(params), _p(cpp_out),
                                        ctypes.c_int64(capacity), ctypes.byref(res), _s(stream)))
    return res


def autotune_entries():
    """The walk autotuner's table: a list of dicts, one per tuned level shape."""
    n = int(lib().nrb_autotune_entries(None, 0))
    arr = (WalkEntry * max(n, 1))()
    n = min(n, int(lib().nrb_autotune_entries(arr, n)))
    out = []
    for e in arr[:n]:
        out.append({"ref_dim": list(e.ref_dim), "cpp_dim": list(e.cpp_dim), "bins": list(e.bins),
                    "objective": {"ty": e.obj_ty, "zchunk": e.obj_zchunk, "resident": e.obj_resident,
                                  "us": e.obj_us, "model_us": e.obj_model_us},
                    "gradient": {"ty": e.grad_ty, "zchunk": e.grad_zchunk, "resident": e.grad_resident,
                                 "us": e.grad_us, "model_us": e.grad_model_us},
                    "candidates": e.candidates})
    return out


def autotune_clear():
    lib().nrb_autotune_clear.restype = None
    lib().nrb_autotune_clear()


def kernel_launch_count() -> int:
    return int(lib().nrb_kernel_launch_count())


def memory_trim(keep_bytes: int = 0):
    """Returns the library pool's unused device memory to the driver, keeping keep_bytes."""
    check(lib().nrb_memory_trim(ctypes.c_size_t(int(keep_bytes))))


def timing_enable(on: bool = True):
    """Brackets every launch of the timed kernels with CUDA events (clears counters)."""
    lib().nrb_timing_enable.restype = None
    lib().nrb_timing_enable(int(bool(on)))


def timing_read(kernel: str):
    """(launches, total device ms, algorithmic bytes) of one timed kernel."""
    n, ms, by = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
    check(lib().nrb_timing_read(kernel.encode(), ctypes.byref(n), ctypes.byref(ms), ctypes.byref(by)))
    return n.value, ms.value, by.value


# ----------------------------------------------------------------------------------------------
# NiftyReg's reg_f3d on the B200 platform (platform/libniftyreg_b200_platform.so,
# include/niftyreg_b200_platform.h)
# ----------------------------------------------------------------------------------------------
PLATFORM_LIB_PATH = os.path.join(HERE, "platform", "libniftyreg_b200_platform.so")
_PLATFORM_LIB = None
PLATFORM_CPU, PLATFORM_B200 = 0, 1


class PlatformParams(ctypes.Structure):
    _fields_ = [("platform", ctypes.c_int32), ("gpu", ctypes.c_int32), ("levels", ctypes.c_int32),
                ("max_iterations", ctypes.c_int32), ("bending_energy", ctypes.c_float),
                ("linear_energy", ctypes.c_float), ("spacing", ctypes.c_float), ("bins", ctypes.c_int32),
                ("verbose", ctypes.c_int32), ("padding", ctypes.c_float)]


class PlatformResult(ctypes.Structure):
    _fields_ = [("cpp_dim", _I3), ("final_nmi", ctypes.c_double), ("objective_evaluations", ctypes.c_int64),
                ("gradient_evaluations", ctypes.c_int64), ("seconds", ctypes.c_double),
                ("level_seconds", ctypes.c_double * 8)]


def platform_available() -> bool:
    """True when the NiftyReg library with the B200 platform has been built (it needs the
    NiftyReg sources: make -C niftyreg_b200/platform)."""
    return os.path.exists(PLATFORM_LIB_PATH)


def platform_lib() -> ctypes.CDLL:
    global _PLATFORM_LIB
    if _PLATFORM_LIB is None:
        if not platform_available():
            raise RuntimeError(f"{PLATFORM_LIB_PATH} is missing: make -C niftyreg_b200/platform "
                               "(NIFTYREG_SOURCE_DIR = the NiftyReg checkout)")
        lib()  # the C ABI it links against, loaded from this package
        L = ctypes.CDLL(PLATFORM_LIB_PATH)
        L.nrb_platform_last_error.restype = ctypes.c_char_p
        _PLATFORM_LIB = L
    return _PLATFORM_LIB


def platform_register(ref: np.ndarray, flo: np.ndarray, pixdim, xyz=None, platform=PLATFORM_B200, levels=1,
                      max_iterations=100, bending_energy=0.005, linear_energy=0.0, spacing=-5.0, bins=64,
                      gpu=-1, verbose=False, padding=math.nan):
    """reg_f3d<float>::Run of NiftyReg's own registration code on the CPU or the B200 platform,
    host volumes [nz, ny, nx] float32 in, (cpp [3, cz, cy, cx], PlatformResult) out."""
    ref = np.ascontiguousarray(ref, np.float32)
    flo = np.ascontiguousarray(flo, np.float32)
    nz, ny, nx = ref.shape
    if xyz is None:
        xyz = identity_header(pixdim)
    xyz = np.ascontiguousarray(xyz, np.float32).ravel()
    p = PlatformParams(int(platform), int(gpu), int(levels), int(max_iterations), float(bending_energy),
                       float(linear_energy), float(spacing), int(bins), int(bool(verbose)), float(padding))
    step = [abs(spacing) * (pixdim[a] if spacing < 0 else 1.0) for a in range(3)]
    cap = 3 * int(np.prod([int(math.ceil(n * pixdim[a] / step[a])) + 8 for a, n in enumerate((nx, ny, nz))]))
    cpp = np.zeros(cap, np.float32)
    res = PlatformResult()
    rc = platform_lib().nrb_platform_f3d_register(
        ref.ctypes.data_as(ctypes.c_void_p), flo.ctypes.data_as(ctypes.c_void_p), _I3(nx, ny, nz),
        _F3(*[float(v) for v in pixdim]), xyz.ctypes.data_as(ctypes.c_void_p), ctypes.byref(p),
        cpp.ctypes.data_as(ctypes.c_void_p), ctypes.c_int64(cap), ctypes.byref(res))
    if rc != 0:
        raise NrbError(-1, platform_lib().nrb_platform_last_error().decode())
    cx, cy, cz = [int(v) for v in res.cpp_dim]
    return cpp[:3 * cx * cy * cz].reshape(3, cz, cy, cx).copy(), res
