// NIfTI-1 single-file images (.nii, .nii.gz) for the request path of a served registration:
// read any scalar or vector image into host float32 with the orientation NiftyReg uses, and write
// float32 results (warped images, control-point grids) that NiftyReg's own tools read back.
//
// Reading follows what reg_io_ReadImageFile does with an image (reg-io/_reg_ReadWriteImage.cpp:
// 51-81): niftilib's header conversion, then reg_checkAndCorrectDimension
// (reg-lib/cpu/_reg_tools.cpp:13-71): singleton axes of zero spacing get spacing 1, a zero
// scl_slope means 1, micron and metre spacings become mm. The voxel -> mm matrix is the sform
// when sform_code > 0, else the qform (quaternion, NIfTI-1 method 2) when qform_code > 0, else
// the spacing on the diagonal: the choice of Content::GetXYZMatrix. Values are converted to float
// and scaled by scl_slope / scl_inter (the reference applies the same scaling inside its intensity
// rescale).
//
// Host code only; no device work and no CUDA calls.
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "niftyreg_b200.h"

namespace nrb {
nrb_status fail(nrb_status s, const std::string& msg);
}

namespace {

// NIfTI-1 header field offsets (the 348-byte layout of the specification)
constexpr int kHdrSize = 348;
constexpr int kOffDim = 40, kOffIntentP1 = 56, kOffIntentCode = 68, kOffDatatype = 70, kOffBitpix = 72;
constexpr int kOffPixdim = 76, kOffVoxOffset = 108, kOffSclSlope = 112, kOffSclInter = 116;
constexpr int kOffXyztUnits = 123, kOffDescrip = 148, kOffQformCode = 252, kOffSformCode = 254;
constexpr int kOffQuatern = 256, kOffSrow = 280, kOffIntentName = 328, kOffMagic = 344;

bool ends_with(const std::string& s, const char *suffix) {
    const size_t n = strlen(suffix);
    return s.size() >= n && s.compare(s.size() - n, n, suffix) == 0;
}

void swap_bytes(unsigned char *p, int n) {
    for (int i = 0; i < n / 2; ++i) std::swap(p[i], p[n - 1 - i]);
}

struct HeaderView {
    std::vector<unsigned char> b;
    bool swap = false;
    template <typename T> T get(int off) const {
        T v;
        unsigned char tmp[sizeof(T)];
        memcpy(tmp, b.data() + off, sizeof(T));
        if (swap) swap_bytes(tmp, sizeof(T));
        memcpy(&v, tmp, sizeof(T));
        return v;
    }
};

// voxel -> mm of a qform: rotation from the unit quaternion (b, c, d; a = sqrt(1 - b2 - c2 - d2),
// renormalised when that is not positive), columns scaled by the spacings, the third by qfac
void quaternion_matrix(double b, double c, double d, double qx, double qy, double qz, double dx, double dy,
                       double dz, double qfac, float m[16]) {
    double a = 1.0 - (b * b + c * c + d * d);
    if (a < 1e-7) {
        const double s = 1.0 / std::sqrt(b * b + c * c + d * d);
        b *= s;
        c *= s;
        d *= s;
        a = 0.0;
    } else {
        a = std::sqrt(a);
    }
    const double sx = dx > 0 ? dx : 1.0, sy = dy > 0 ? dy : 1.0;
    double sz = dz > 0 ? dz : 1.0;
    if (qfac < 0) sz = -sz;
    const double r[3][3] = { { a * a + b * b - c * c - d * d, 2.0 * (b * c - a * d), 2.0 * (b * d + a * c) },
                             { 2.0 * (b * c + a * d), a * a + c * c - b * b - d * d, 2.0 * (c * d - a * b) },
                             { 2.0 * (b * d - a * c), 2.0 * (c * d + a * b), a * a + d * d - c * c - b * b } };
    const double s[3] = { sx, sy, sz }, t[3] = { qx, qy, qz };
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) m[4 * i + j] = (float)(r[i][j] * s[j]);
        m[4 * i + 3] = (float)t[i];
    }
    m[12] = m[13] = m[14] = 0.f;
    m[15] = 1.f;
}

// inverse of an affine voxel <-> mm matrix, in double
bool affine_inverse(const float m[16], float out[16]) {
    double a[3][3], t[3];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) a[i][j] = m[4 * i + j];
        t[i] = m[4 * i + 3];
    }
    const double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
                       a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                       a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    if (det == 0.0 || !std::isfinite(det)) return false;
    double inv[3][3];
    inv[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) / det;
    inv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
    inv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
    inv[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) / det;
    inv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
    inv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
    inv[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) / det;
    inv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
    inv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        for (int j = 0; j < 3; ++j) {
            out[4 * i + j] = (float)inv[i][j];
            s += inv[i][j] * t[j];
        }
        out[4 * i + 3] = (float)-s;
    }
    out[12] = out[13] = out[14] = 0.f;
    out[15] = 1.f;
    return true;
}

// the whole file through zlib (which reads uncompressed files as they are)
bool read_all(const char *path, std::vector<unsigned char>& out) {
    gzFile f = gzopen(path, "rb");
    if (!f) return false;
    unsigned char buf[1 << 16];
    int n;
    while ((n = gzread(f, buf, sizeof buf)) > 0) out.insert(out.end(), buf, buf + n);
    const bool ok = n == 0;
    gzclose(f);
    return ok;
}

template <typename T>
void convert(const unsigned char *src, size_t n, bool swap, float slope, float inter, float *dst) {
    const bool scale = !(slope == 1.f && inter == 0.f);
    for (size_t i = 0; i < n; ++i) {
        unsigned char tmp[sizeof(T)];
        memcpy(tmp, src + i * sizeof(T), sizeof(T));
        if (swap) swap_bytes(tmp, sizeof(T));
        T v;
        memcpy(&v, tmp, sizeof(T));
        const float f = (float)v;
        dst[i] = scale ? (float)((double)f * slope + inter) : f;
    }
}

}  // namespace

using nrb::fail;

extern "C" nrb_status nrb_image_read(const char *path, nrb_image *out) {
    if (!path || !out) return fail(NRB_ERR_INVALID, "nrb_image_read: null pointer");
    memset(out, 0, sizeof(*out));
    const std::string p(path);
    if (!ends_with(p, ".nii") && !ends_with(p, ".nii.gz"))
        return fail(NRB_ERR_UNSUPPORTED, "nrb_image_read: only single-file NIfTI-1 (.nii, .nii.gz) is read");
    std::vector<unsigned char> file;
    if (!read_all(path, file)) return fail(NRB_ERR_INVALID, "nrb_image_read: cannot read " + p);
    if (file.size() < (size_t)kHdrSize) return fail(NRB_ERR_INVALID, "nrb_image_read: file shorter than a NIfTI-1 header");
    HeaderView h;
    h.b.assign(file.begin(), file.begin() + kHdrSize);
    if (h.get<int32_t>(0) != kHdrSize) {
        h.swap = true;
        if (h.get<int32_t>(0) != kHdrSize) return fail(NRB_ERR_INVALID, "nrb_image_read: not a NIfTI-1 header");
    }
    if (memcmp(h.b.data() + kOffMagic, "n+1", 4) != 0)
        return fail(NRB_ERR_UNSUPPORTED, "nrb_image_read: not a single-file NIfTI-1 image (magic n+1)");
    int dim[8];
    for (int i = 0; i < 8; ++i) dim[i] = h.get<int16_t>(kOffDim + 2 * i);
    if (dim[0] < 1 || dim[0] > 7) return fail(NRB_ERR_INVALID, "nrb_image_read: dim[0] outside [1, 7]");
    for (int i = dim[0] + 1; i < 8; ++i) dim[i] = 1;
    for (int i = 1; i <= dim[0]; ++i)
        if (dim[i] < 1) dim[i] = 1;
    float pix[8];
    for (int i = 0; i < 8; ++i) pix[i] = h.get<float>(kOffPixdim + 4 * i);
    const int datatype = h.get<int16_t>(kOffDatatype);
    const float vox_offset = h.get<float>(kOffVoxOffset);
    float slope = h.get<float>(kOffSclSlope);
    const float inter = h.get<float>(kOffSclInter);
    if (slope == 0.f || !std::isfinite(slope)) slope = 1.f;
    const float inter_v = std::isfinite(inter) ? inter : 0.f;
    const int qform_code = h.get<int16_t>(kOffQformCode), sform_code = h.get<int16_t>(kOffSformCode);

    // orientation: sform, else qform, else the spacings (with the spacings as read)
    float xyz[16];
    if (sform_code > 0) {
        for (int i = 0; i < 12; ++i) xyz[i] = h.get<float>(kOffSrow + 4 * i);
        xyz[12] = xyz[13] = xyz[14] = 0.f;
        xyz[15] = 1.f;
    } else if (qform_code > 0) {
        quaternion_matrix(h.get<float>(kOffQuatern), h.get<float>(kOffQuatern + 4), h.get<float>(kOffQuatern + 8),
                          h.get<float>(kOffQuatern + 12), h.get<float>(kOffQuatern + 16),
                          h.get<float>(kOffQuatern + 20), pix[1], pix[2], pix[3], pix[0] < 0 ? -1.0 : 1.0, xyz);
    } else {
        quaternion_matrix(0, 0, 0, 0, 0, 0, pix[1], pix[2], pix[3], 1.0, xyz);
    }
    // spacing corrections of reg_checkAndCorrectDimension (the matrix keeps what was read)
    if (dim[2] == 1 && pix[2] == 0.f) pix[2] = 1.f;
    if (dim[3] == 1 && pix[3] == 0.f) pix[3] = 1.f;
    const int units = h.b[kOffXyztUnits] & 0x07;
    if (units == 3)
        for (int d = 1; d <= 3; ++d) pix[d] /= 1000.f;
    if (units == 1)
        for (int d = 1; d <= 3; ++d) pix[d] *= 1000.f;

    // element counts: each dim is at most 32767, so the products are checked for overflow before
    // any size is derived from them, and bounded by the file's length below
    size_t nvox3 = 1, nvol = 1;
    bool overflow = false;
    for (int i = 1; i <= 3; ++i) overflow |= __builtin_mul_overflow(nvox3, (size_t)dim[i], &nvox3);
    for (int i = 4; i < 8; ++i) overflow |= __builtin_mul_overflow(nvol, (size_t)dim[i], &nvol);
    size_t n = 0;
    overflow |= __builtin_mul_overflow(nvox3, nvol, &n);
    if (overflow) return fail(NRB_ERR_INVALID, "nrb_image_read: voxel count overflows");
    if (nvol > (size_t)INT32_MAX) return fail(NRB_ERR_INVALID, "nrb_image_read: more than 2^31 - 1 volumes");
    int bytes = 0;
    switch (datatype) {
    case 2: case 256: bytes = 1; break;     // uint8, int8
    case 4: case 512: bytes = 2; break;     // int16, uint16
    case 8: case 16: case 768: bytes = 4; break;  // int32, float32, uint32
    case 64: case 1024: case 1280: bytes = 8; break;  // float64, int64, uint64
    default:
        return fail(NRB_ERR_UNSUPPORTED, "nrb_image_read: datatype " + std::to_string(datatype) +
                                              " (complex, RGB or unknown) is not read");
    }
    if (!std::isfinite(vox_offset) || vox_offset >= (float)file.size())
        return fail(NRB_ERR_INVALID, "nrb_image_read: vox_offset is not finite or lies past the end of the file");
    const size_t start = vox_offset > 0 ? (size_t)vox_offset : 352;
    // n <= (file length - start) / bytes bounds n * bytes and n * sizeof(float) far below 2^64
    if (start > file.size() || n > (file.size() - start) / (size_t)bytes)
        return fail(NRB_ERR_INVALID, "nrb_image_read: data shorter than the header says");
    float *data = (float *)malloc(std::max<size_t>(n, 1) * sizeof(float));
    if (!data) return fail(NRB_ERR_OOM, "nrb_image_read: host allocation failed");
    const unsigned char *src = file.data() + start;
    switch (datatype) {
    case 2: convert<uint8_t>(src, n, h.swap, slope, inter_v, data); break;
    case 256: convert<int8_t>(src, n, h.swap, slope, inter_v, data); break;
    case 4: convert<int16_t>(src, n, h.swap, slope, inter_v, data); break;
    case 512: convert<uint16_t>(src, n, h.swap, slope, inter_v, data); break;
    case 8: convert<int32_t>(src, n, h.swap, slope, inter_v, data); break;
    case 768: convert<uint32_t>(src, n, h.swap, slope, inter_v, data); break;
    case 16: convert<float>(src, n, h.swap, slope, inter_v, data); break;
    case 64: convert<double>(src, n, h.swap, slope, inter_v, data); break;
    case 1024: convert<int64_t>(src, n, h.swap, slope, inter_v, data); break;
    case 1280: convert<uint64_t>(src, n, h.swap, slope, inter_v, data); break;
    }
    for (int i = 0; i < 3; ++i) {
        out->dim[i] = dim[i + 1];
        out->pixdim[i] = pix[i + 1];
    }
    out->nvol = (int32_t)nvol;
    memcpy(out->xyz, xyz, sizeof xyz);
    if (!affine_inverse(xyz, out->ijk)) {
        free(data);
        return fail(NRB_ERR_INVALID, "nrb_image_read: singular voxel-to-mm matrix");
    }
    out->sform_code = sform_code > 0 ? sform_code : 0;
    out->qform_code = qform_code > 0 ? qform_code : 0;
    out->intent_code = h.get<int16_t>(kOffIntentCode);
    out->intent_p1 = h.get<float>(kOffIntentP1);
    out->intent_p2 = h.get<float>(kOffIntentP1 + 4);
    memcpy(out->intent_name, h.b.data() + kOffIntentName, 16);
    out->intent_name[15] = 0;
    out->data = data;
    return NRB_OK;
}

extern "C" void nrb_image_free(nrb_image *img) {
    if (!img) return;
    free(img->data);
    img->data = nullptr;
}

extern "C" nrb_status nrb_image_write(const char *path, const nrb_image *img) {
    if (!path || !img || !img->data) return fail(NRB_ERR_INVALID, "nrb_image_write: null pointer");
    const std::string p(path);
    const bool gz = ends_with(p, ".nii.gz");
    if (!gz && !ends_with(p, ".nii"))
        return fail(NRB_ERR_UNSUPPORTED, "nrb_image_write: only single-file NIfTI-1 (.nii, .nii.gz) is written");
    for (int i = 0; i < 3; ++i)
        if (img->dim[i] < 1 || img->dim[i] > 32767 || !(img->pixdim[i] > 0))
            return fail(NRB_ERR_INVALID, "nrb_image_write: dims in [1, 32767] and positive spacings expected");
    if (img->nvol < 1 || img->nvol > 32767) return fail(NRB_ERR_INVALID, "nrb_image_write: nvol in [1, 32767] expected");
    unsigned char hdr[352];
    memset(hdr, 0, sizeof hdr);
    auto put = [&](int off, const void *v, size_t n) { memcpy(hdr + off, v, n); };
    const int32_t hs = kHdrSize;
    put(0, &hs, 4);
    hdr[38] = 'r';  // "regular"
    int16_t dim[8] = { 3, (int16_t)img->dim[0], (int16_t)img->dim[1], (int16_t)img->dim[2], 1, 1, 1, 1 };
    if (img->nvol > 1) {
        dim[0] = 5;  // vector images: the components along the 5th axis, as NiftyReg stores them
        dim[5] = (int16_t)img->nvol;
    }
    put(kOffDim, dim, sizeof dim);
    put(kOffIntentP1, &img->intent_p1, 4);
    put(kOffIntentP1 + 4, &img->intent_p2, 4);
    const int16_t intent = (int16_t)img->intent_code, datatype = 16, bitpix = 32;
    put(kOffIntentCode, &intent, 2);
    put(kOffDatatype, &datatype, 2);
    put(kOffBitpix, &bitpix, 2);
    const float pix[8] = { 1.f, img->pixdim[0], img->pixdim[1], img->pixdim[2], 1.f, 1.f, 1.f, 1.f };
    put(kOffPixdim, pix, sizeof pix);
    const float vox_offset = 352.f, slope = 1.f;
    put(kOffVoxOffset, &vox_offset, 4);
    put(kOffSclSlope, &slope, 4);
    hdr[kOffXyztUnits] = 2;  // mm
    const char descrip[] = "niftyreg_b200";
    put(kOffDescrip, descrip, sizeof descrip);
    const int16_t qcode = 0,
                  scode = (int16_t)(img->sform_code > 0 ? img->sform_code : img->qform_code > 0 ? img->qform_code : 1);
    put(kOffQformCode, &qcode, 2);
    put(kOffSformCode, &scode, 2);
    put(kOffSrow, img->xyz, 12 * sizeof(float));
    char name[16];
    memcpy(name, img->intent_name, 16);
    name[15] = 0;
    put(kOffIntentName, name, 16);
    put(kOffMagic, "n+1", 4);
    const size_t n = (size_t)img->dim[0] * img->dim[1] * img->dim[2] * img->nvol;
    bool ok;
    if (gz) {
        gzFile f = gzopen(path, "wb6");
        if (!f) return fail(NRB_ERR_INVALID, "nrb_image_write: cannot open " + p);
        ok = gzwrite(f, hdr, sizeof hdr) == (int)sizeof hdr;
        const char *src = (const char *)img->data;
        size_t left = n * sizeof(float);
        while (ok && left > 0) {
            const unsigned chunk = (unsigned)std::min<size_t>(left, 1u << 30);
            ok = gzwrite(f, src, chunk) == (int)chunk;
            src += chunk;
            left -= chunk;
        }
        ok = (gzclose(f) == Z_OK) && ok;
    } else {
        FILE *f = fopen(path, "wb");
        if (!f) return fail(NRB_ERR_INVALID, "nrb_image_write: cannot open " + p);
        ok = fwrite(hdr, 1, sizeof hdr, f) == sizeof hdr && fwrite(img->data, sizeof(float), n, f) == n;
        ok = (fclose(f) == 0) && ok;
    }
    return ok ? NRB_OK : fail(NRB_ERR_INVALID, "nrb_image_write: write failed for " + p);
}
