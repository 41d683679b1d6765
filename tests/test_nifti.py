"""NIfTI-1 I/O of the request path (nrb_image_read / nrb_image_write), CPU only.

Files are built byte by byte from the NIfTI-1 layout, so every header case is explicit: integer
and real datatypes with scl_slope / scl_inter, both byte orders, sform, qform (quaternion with
qfac -1), neither form, micron units, a zero spacing on a singleton axis, vector images, gzip.
The reader must give what NiftyReg's own reader gives on the same file (niftilib +
reg_checkAndCorrectDimension, through oracle/_ref): same dims, spacings and data bit for bit,
and the same voxel -> mm matrix (within 1e-6: the quaternion rotation is evaluated in another
order). Files the library writes must read back, through the reference's reader too.
"""
import gzip
import struct

import numpy as np
import pytest

import niftyreg_b200 as nrb
import oracle
from tests.helpers import ensure_built

DTYPES = {2: "u1", 4: "i2", 8: "i4", 16: "f4", 64: "f8", 256: "i1", 512: "u2", 768: "u4"}


def nifti_bytes(data, dtype_code, pixdim=(1.0, 1.0, 1.0), big_endian=False, slope=1.0, inter=0.0, sform=None,
                qform=None, qfac=1.0, units=2, dim_extra=(), pixdim0_zero_axis=None):
    """A single-file NIfTI-1 image: data is [..., nz, ny, nx] (extra leading axes become dims 4+)."""
    e = ">" if big_endian else "<"
    a = np.asarray(data)
    nz, ny, nx = a.shape[-3:]
    lead = list(a.shape[:-3])[::-1]
    dims = [3 + len(lead), nx, ny, nz] + lead
    dims += [1] * (8 - len(dims))
    pix = [qfac, *pixdim] + [1.0] * 4
    if pixdim0_zero_axis is not None:
        pix[pixdim0_zero_axis] = 0.0
    h = bytearray(352)
    struct.pack_into(e + "i", h, 0, 348)
    struct.pack_into(e + "8h", h, 40, *dims)
    struct.pack_into(e + "h", h, 70, dtype_code)
    struct.pack_into(e + "h", h, 72, np.dtype(DTYPES[dtype_code]).itemsize * 8)
    struct.pack_into(e + "8f", h, 76, *pix)
    struct.pack_into(e + "f", h, 108, 352.0)
    struct.pack_into(e + "2f", h, 112, slope, inter)
    h[123] = units
    if qform is not None:
        b, c, d, qx, qy, qz = qform
        struct.pack_into(e + "h", h, 252, 1)
        struct.pack_into(e + "6f", h, 256, b, c, d, qx, qy, qz)
    if sform is not None:
        struct.pack_into(e + "h", h, 254, 2)
        struct.pack_into(e + "12f", h, 280, *np.asarray(sform, np.float32).reshape(4, 4)[:3].ravel())
    h[344:348] = b"n+1\0"
    body = np.ascontiguousarray(a, dtype=np.dtype(DTYPES[dtype_code]).newbyteorder(e)).tobytes()
    return bytes(h) + body


CASES = {
    "int16_slope": dict(dtype_code=4, slope=0.5, inter=-3.0),
    "uint8": dict(dtype_code=2),
    "int32_big_endian": dict(dtype_code=8, big_endian=True),
    "float64_sform": dict(dtype_code=64, sform=[[0.9, 0.1, 0.0, -20.0], [-0.1, 0.95, 0.05, 12.5],
                                                 [0.0, -0.05, 1.4, 3.0], [0, 0, 0, 1]]),
    "float32_qform_qfac": dict(dtype_code=16, qform=(0.1, -0.2, 0.3, 5.0, -6.0, 7.0), qfac=-1.0,
                               pixdim=(1.1, 0.8, 1.7)),
    "int8_no_form": dict(dtype_code=256, pixdim=(2.0, 1.5, 1.25)),
    "uint16_micron": dict(dtype_code=512, units=3, pixdim=(500.0, 500.0, 800.0)),
    "uint32_both_forms": dict(dtype_code=768, qform=(0.0, 0.0, 0.7071068, 1.0, 2.0, 3.0),
                              sform=[[1.0, 0, 0, 1.0], [0, 1.0, 0, 2.0], [0, 0, 1.0, 3.0], [0, 0, 0, 1]]),
}


def make_data(dtype_code, shape, seed):
    rng = np.random.default_rng(seed)
    dt = np.dtype(DTYPES[dtype_code])
    if dt.kind == "f":
        return rng.normal(100, 40, shape).astype(dt)
    info = np.iinfo(dt)
    return rng.integers(max(info.min, -30000), min(info.max, 30000), shape, endpoint=True).astype(dt)


@pytest.fixture(scope="module")
def R():
    ensure_built()
    if not oracle.ref_available():
        pytest.skip("oracle/_ref (the reference build) is not present")
    return oracle.Ref()


@pytest.mark.parametrize("name", sorted(CASES))
def test_reader_matches_the_reference_reader(R, tmp_path, name):
    kw = CASES[name]
    data = make_data(kw["dtype_code"], (6, 7, 9), seed=len(name))
    p = tmp_path / f"{name}.nii"
    p.write_bytes(nifti_bytes(data, **kw))
    ours, pix, xyz = nrb.read_image(p)
    dim, nvol, rpix, rxyz, rdata = R.image_read(p)
    assert list(dim) == [9, 7, 6] and nvol == 1 and ours.shape == (1, 6, 7, 9)
    assert np.array_equal(np.asarray(pix, np.float32), rpix)
    assert np.allclose(xyz, rxyz, rtol=1e-6, atol=1e-5)
    assert np.array_equal(ours.ravel(), rdata)


def test_vector_image_and_zero_spacing_on_a_singleton_axis(R, tmp_path):
    data = np.random.default_rng(3).normal(size=(3, 1, 5, 8)).astype(np.float32)  # nu = 3, nz = 1
    p = tmp_path / "vec.nii"
    raw = bytearray(nifti_bytes(data[:, None], 16, pixdim=(1.0, 2.0, 1.0), pixdim0_zero_axis=3))
    struct.pack_into("<8h", raw, 40, 5, 8, 5, 1, 1, 3, 1, 1)  # nx, ny, nz, nt, nu
    p.write_bytes(bytes(raw))
    ours, pix, _ = nrb.read_image(p)
    dim, nvol, rpix, _, rdata = R.image_read(p)
    assert nvol == 3 and ours.shape == (3, 1, 5, 8)
    assert pix[2] == 1.0 and np.array_equal(np.asarray(pix, np.float32), rpix)
    assert np.array_equal(ours.ravel(), rdata)


def test_gzip_reads_like_the_plain_file(tmp_path):
    ensure_built()
    data = make_data(4, (5, 6, 7), seed=5)
    raw = nifti_bytes(data, 4, slope=2.0, inter=1.0)
    (tmp_path / "a.nii").write_bytes(raw)
    (tmp_path / "a.nii.gz").write_bytes(gzip.compress(raw))
    a, pa, xa = nrb.read_image(tmp_path / "a.nii")
    b, pb, xb = nrb.read_image(tmp_path / "a.nii.gz")
    assert np.array_equal(a, b) and pa == pb and np.array_equal(xa, xb)
    assert np.array_equal(a[0], (data.astype(np.float32).astype(np.float64) * 2.0 + 1.0).astype(np.float32))


def test_written_files_read_back_here_and_in_the_reference(R, tmp_path):
    rng = np.random.default_rng(6)
    data = rng.normal(size=(3, 6, 5, 4)).astype(np.float32)
    xyz = np.array([[5.0, 0, 0, -5.0], [0, 5.0, 0, -5.0], [0, 0, 5.0, -5.0], [0, 0, 0, 1]], np.float32)
    for name in ("grid.nii", "grid.nii.gz"):
        p = tmp_path / name
        nrb.write_image(p, data, (5.0, 5.0, 5.0), xyz, intent_code=1007, intent_p1=2.0, intent_name=b"NREG_TRANS")
        back, pix, bxyz = nrb.read_image(p)
        assert np.array_equal(back, data) and pix == (5.0, 5.0, 5.0) and np.array_equal(bxyz, xyz)
    dim, nvol, rpix, rxyz, rdata = R.image_read(tmp_path / "grid.nii")
    assert list(dim) == [4, 5, 6] and nvol == 3
    assert np.array_equal(rxyz, xyz) and np.array_equal(rdata, data.ravel())


def test_refusals(tmp_path):
    ensure_built()
    with pytest.raises(nrb.NrbError):
        nrb.read_image(tmp_path / "missing.nii")
    (tmp_path / "bad.nii").write_bytes(b"\0" * 400)
    with pytest.raises(nrb.NrbError):
        nrb.read_image(tmp_path / "bad.nii")
    with pytest.raises(nrb.NrbError):
        nrb.read_image(tmp_path / "x.hdr")
    data = np.zeros((2, 2, 2), np.float32)
    raw = bytearray(nifti_bytes(data, 16))
    struct.pack_into("<h", raw, 70, 32)  # complex64
    (tmp_path / "complex.nii").write_bytes(bytes(raw))
    with pytest.raises(nrb.NrbError):
        nrb.read_image(tmp_path / "complex.nii")


def test_headers_whose_sizes_overflow_or_point_past_the_file_are_refused(tmp_path):
    """Crafted headers: element counts whose byte size wraps 64 bits, a vox_offset that is NaN or
    past the end of the file, and data shorter than the dims say are all refused before any
    allocation sized from them."""
    ensure_built()
    data = np.zeros((2, 2, 2), np.float32)
    base = bytearray(nifti_bytes(data, 16))

    def refused(name, raw):
        (tmp_path / name).write_bytes(bytes(raw))
        with pytest.raises(nrb.NrbError):
            nrb.read_image(tmp_path / name)

    # 16384^4 * 64 voxels = 2^62: times 4 bytes wraps to 0 in 64-bit arithmetic
    wrap = bytearray(base)
    struct.pack_into("<8h", wrap, 40, 5, 16384, 16384, 16384, 16384, 64, 1, 1)
    refused("wrap.nii", wrap)
    # every dim at its maximum: the element count itself overflows
    huge = bytearray(base)
    struct.pack_into("<8h", huge, 40, 7, 32767, 32767, 32767, 32767, 32767, 32767, 32767)
    refused("huge.nii", huge)
    for off in (float("nan"), float("inf"), 1.0e9):
        raw = bytearray(base)
        struct.pack_into("<f", raw, 108, off)
        refused(f"offset_{off}.nii", raw)
    short = bytearray(base)
    struct.pack_into("<8h", short, 40, 3, 2, 2, 3, 1, 1, 1, 1)  # 12 voxels, the file holds 8
    refused("short.nii", short)
    # the unmodified file still reads
    (tmp_path / "ok.nii").write_bytes(bytes(base))
    nrb.read_image(tmp_path / "ok.nii")
