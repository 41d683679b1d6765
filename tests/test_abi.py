"""The C ABI: the shared library builds for sm_100a, loads without a GPU, exports every
function include/niftyreg_b200.h declares, and host-only entry points behave."""
import ctypes
import os
import re
import subprocess

import numpy as np

import niftyreg_b200 as nrb
from tests.helpers import ROOT, ArgBuffers, ensure_built


def declared_functions():
    text = open(os.path.join(ROOT, "include", "niftyreg_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nrb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    ensure_built()
    lib = nrb.lib()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_library_is_sm100a_only():
    ensure_built()
    out = os.popen(f"/usr/local/cuda/bin/cuobjdump --list-elf {nrb.LIB_PATH} 2>/dev/null").read()
    archs = set(re.findall(r"sm_(\d+a?)", out))
    assert archs == {"100a"}, archs


def test_host_entry_points_without_gpu():
    ensure_built()
    p = nrb.default_params()
    assert p.levels == 3 and p.max_iterations == 150 and abs(p.bending_energy - 0.001) < 1e-9
    assert np.isnan(p.padding) and p.ref_bins == 64
    p = nrb.default_params(spacing=(-5.0,))
    # reg_createControlPointGrid: ceil(n * d / s + 3)
    assert nrb.grid_dims((182, 218, 182), (1.0, 1.0, 1.0), p) == [40, 47, 40]
    assert nrb.grid_dims((64, 64, 64), (1.0, 1.0, 1.0), p) == [16, 16, 16]
    assert nrb.grid_dims((512, 512, 320), (0.8, 0.8, 1.5), nrb.default_params(spacing=(10.0,))) == [44, 44, 51]
    assert p.autotune == 1 and p.floating_texture == 1
    # the walk table is host state: empty until a registration tunes a shape
    nrb.autotune_clear()
    assert nrb.autotune_entries() == []


def test_invalid_arguments_are_reported():
    ensure_built()
    lib = nrb.lib()
    out = ctypes.c_void_p()
    assert lib.nrb_nmi_create(2, 68, ctypes.byref(out)) == 1  # NRB_ERR_INVALID
    assert b"bins" in lib.nrb_last_error()
    assert lib.nrb_get_deformation_field(None, None, None, None, None) == 1
    # interpolation orders other than 0, 1 and 3 are refused before any device work
    g = nrb.make_geometry((8, 8, 8), (1.0, 1.0, 1.0), nrb.identity_header((1.0, 1.0, 1.0)), (8, 8, 8), (1.0, 1.0, 1.0),
                          nrb.identity_header((1.0, 1.0, 1.0)), (5, 5, 5), (5.0, 5.0, 5.0),
                          nrb.identity_header((5.0, 5.0, 5.0), (-5.0, -5.0, -5.0)))
    fake = ArgBuffers(1)[0]  # a real buffer: the order check comes first
    assert lib.nrb_resample_image_order(ctypes.byref(g), fake, fake, None, 2, ctypes.c_float(0.0), fake, None) == 2
    assert b"order" in lib.nrb_last_error()
    assert lib.nrb_f3d_warped_image(ctypes.byref(g), fake, fake, 4, ctypes.c_float(0.0), fake, None) == 2


def test_f3d2_refusals_before_any_device_work(tmp_path):
    """The velocity-field entry points check their arguments before touching the device."""
    ensure_built()
    lib = nrb.lib()
    bufs = ArgBuffers(2)  # real buffers: every check below comes first
    fake = bufs[0]
    eye = nrb.identity_header((1.0, 1.0, 1.0))
    x16 = (ctypes.c_float * 16)(*[float(v) for v in eye.ravel()])
    dim = (ctypes.c_int32 * 3)(4, 4, 4)
    # composition in place over the applied field itself
    assert lib.nrb_def_field_compose(dim, x16, x16, fake, fake, None) == 1
    assert b"alias" in lib.nrb_last_error()
    flat = nrb.make_geometry((8, 8, 1), (1.0, 1.0, 1.0), eye, (8, 8, 1), (1.0, 1.0, 1.0), eye, (5, 5, 4),
                             (5.0, 5.0, 5.0), nrb.identity_header((5.0, 5.0, 5.0), (-5.0, -5.0, -5.0)))
    # the Jacobian's finite differences need two voxels per axis
    assert lib.nrb_exponentiate_gradient(ctypes.byref(flat), fake, 6, fake, None) == 1
    g = nrb.make_geometry((8, 8, 8), (1.0, 1.0, 1.0), eye, (8, 8, 8), (1.0, 1.0, 1.0), eye, (5, 5, 5),
                          (5.0, 5.0, 5.0), nrb.identity_header((5.0, 5.0, 5.0), (-5.0, -5.0, -5.0)))
    assert lib.nrb_exponentiate_gradient(ctypes.byref(g), fake, 0, fake, None) == 1
    steps = ctypes.c_int32(-1)
    assert lib.nrb_get_def_field_from_velocity_grid(ctypes.byref(g), fake, 0, ctypes.byref(steps), fake, None) == 1
    other = nrb.make_geometry((8, 8, 8), (1.0, 1.0, 1.0), eye, (8, 8, 8), (1.0, 1.0, 1.0), eye, (6, 5, 5),
                              (5.0, 5.0, 5.0), nrb.identity_header((5.0, 5.0, 5.0), (-5.0, -5.0, -5.0)))
    assert lib.nrb_symmetrise_velocity_fields(ctypes.byref(g), fake, ctypes.byref(other), bufs[1],
                                              None) == 1
    assert lib.nrb_symmetrise_velocity_fields(ctypes.byref(g), fake, ctypes.byref(g), fake, None) == 1
    # images and files: checked on the host
    params = nrb.default_params(levels=1, max_iterations=2)
    assert lib.nrb_f3d2_register_images(None, None, ctypes.byref(params), None, None, None, None, None) == 1
    missing = str(tmp_path / "missing.nii").encode()
    assert lib.nrb_f3d2_register_files(missing, missing, ctypes.byref(params), str(tmp_path / "c.nii").encode(),
                                       None, None) != 0


def test_footprint_is_host_only_and_monotone():
    """Admission unit of the server: computed on the host, grows with the volume, and covers at
    least the resident pyramid (2 images x 4 bytes x the finest level)."""
    ensure_built()
    p = nrb.default_params(levels=2, spacing=(-5.0,))
    assert p.host_loop == 0
    sizes = [(64, 64, 64), (128, 128, 96), (182, 218, 182), (256, 256, 256)]
    fps = [nrb.footprint(d, (1.0, 1.0, 1.0), p) for d in sizes]
    assert fps == sorted(fps)
    for d, f in zip(sizes, fps):
        n = d[0] * d[1] * d[2]
        assert 8 * n < f < 80 * n + (8 << 20)
    # the padded floating copy (4 bytes per voxel of the volume grown by the margin) is part of
    # a level's working set
    assert p.floating_margin == 8
    d = (64, 64, 64)
    p0 = nrb.default_params(levels=2, spacing=(-5.0,), floating_margin=0)
    assert 0 < nrb.footprint(d, (1.0, 1.0, 1.0), p) - nrb.footprint(d, (1.0, 1.0, 1.0), p0) <= 4 * 80 ** 3


def test_library_has_no_undefined_internal_symbols():
    """Every function of the library's own namespace that one translation unit calls is defined
    in another: the shared library links without them, so a missing definition would only show
    when the first call fails to resolve."""
    ensure_built()
    out = subprocess.run(["nm", "-C", "-u", nrb.LIB_PATH], capture_output=True, text=True, check=True).stdout
    missing = [l.strip() for l in out.splitlines() if "nrb::" in l]
    assert not missing, missing
