/* Test infrastructure only (the checker; never linked into the product).
 *
 * Plain-C restatement of the reference NiftyReg CPU algorithm on the F3D objective-and-gradient
 * path. Each function cites the reference file:line (paths relative to the NiftyReg source
 * tree) whose arithmetic it restates. Where the reference has an SSE and a scalar variant, the
 * scalar evaluation order is restated; parity with the SSE build is a tolerance question. */
#include "nrb_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

static size_t nvox3(const int d[3]) { return (size_t)d[0] * d[1] * d[2]; }

/* Mat44Mul, reg-lib/cpu/Maths.hpp:272-286: evaluated in double, rounded to float */
static void mat44_apply(const float m[16], const float in[3], float out[3]) {
    for (int i = 0; i < 3; ++i)
        out[i] = (float)((double)m[4 * i + 0] * in[0] + (double)m[4 * i + 1] * in[1]
                         + (double)m[4 * i + 2] * in[2] + (double)m[4 * i + 3]);
}

/* reg-lib/cpu/_reg_splineBasis.cpp:17-26 */
void orc_bspline_basis(float t, float b[4]) {
    const float ff = t * t, fff = ff * t, mf = (float)(1.0 - t);
    b[0] = (float)(mf * mf * mf / 6.0);
    b[1] = (float)((3.0 * fff - 6.0 * ff + 4.0) / 6.0);
    b[2] = (float)((-3.0 * fff + 3.0 * ff + 3.0 * t + 1.0) / 6.0);
    b[3] = (float)(fff / 6.0);
}

/* Cubic B-spline deformation field (positions in mm) from a control-point grid whose node 0
 * sits one spacing before voxel 0: generic branch of reg_cubic_spline_getDeformationField3D,
 * reg-lib/cpu/_reg_localTrans.cpp:1079-1084 (gridVoxelSpacing) and :1305-1453 (per voxel
 * xPre = int(x/s), basis = x/s - xPre, 64-term sum in (c, b, a) order). Masked voxels get 0. */
int orc_deformation_field(const float *cpp, const int cdim[3], const float cpix[3],
                          const int rdim[3], const float rpix[3], const int *mask, float *def) {
    const size_t nc = nvox3(cdim), nr = nvox3(rdim);
    const float gs[3] = { cpix[0] / rpix[0], cpix[1] / rpix[1], cpix[2] / rpix[2] };
    const float *cx = cpp, *cy = cpp + nc, *cz = cpp + 2 * nc;
    float *dx = def, *dy = def + nr, *dz = def + 2 * nr;
    for (int z = 0; z < rdim[2]; ++z) {
        const int zPre = (int)((float)z / gs[2]);
        float bz[4];
        float t = (float)z / gs[2] - (float)zPre;
        if (t < 0) t = 0;
        orc_bspline_basis(t, bz);
        for (int y = 0; y < rdim[1]; ++y) {
            const int yPre = (int)((float)y / gs[1]);
            float by[4], yz[16];
            t = (float)y / gs[1] - (float)yPre;
            if (t < 0) t = 0;
            orc_bspline_basis(t, by);
            for (int c = 0; c < 4; ++c)
                for (int b = 0; b < 4; ++b) yz[4 * c + b] = by[b] * bz[c];
            for (int x = 0; x < rdim[0]; ++x) {
                const size_t idx = ((size_t)z * rdim[1] + y) * rdim[0] + x;
                const int xPre = (int)((float)x / gs[0]);
                float bx[4];
                t = (float)x / gs[0] - (float)xPre;
                if (t < 0) t = 0;
                orc_bspline_basis(t, bx);
                float p[3] = { 0, 0, 0 };
                if (!mask || mask[idx] > -1) {
                    for (int c = 0; c < 4; ++c)
                        for (int b = 0; b < 4; ++b)
                            for (int a = 0; a < 4; ++a) {
                                const int X = xPre + a, Y = yPre + b, Z = zPre + c;
                                if (X < 0 || Y < 0 || Z < 0 || X >= cdim[0] || Y >= cdim[1] || Z >= cdim[2])
                                    return -1; /* outside the grid support: not an F3D layout */
                                const size_t ci = ((size_t)Z * cdim[1] + Y) * cdim[0] + X;
                                const float w = bx[a] * yz[4 * c + b];
                                p[0] += cx[ci] * w;
                                p[1] += cy[ci] * w;
                                p[2] += cz[ci] * w;
                            }
                }
                dx[idx] = p[0];
                dy[idx] = p[1];
                dz[idx] = p[2];
            }
        }
    }
    return 0;
}

/* Trilinear warp with padding: ResampleImage3D, reg-lib/cpu/_reg_resampling.cpp:316-464 with
 * the linear kernel of :79-83. A tap outside the floating volume contributes padding*basis, so
 * NaN padding turns every border voxel into NaN even where that tap's weight is 0. Voxels
 * outside the mask are left untouched. */
int orc_resample_linear(const float *flo, const int fdim[3], const float flo_ijk[16],
                        const float *def, const int rdim[3], const int *mask, float pad,
                        float *warped) {
    const size_t nr = nvox3(rdim);
    for (size_t i = 0; i < nr; ++i) {
        if (mask && mask[i] <= -1) continue;
        const float world[3] = { def[i], def[nr + i], def[2 * nr + i] };
        float pos[3];
        mat44_apply(flo_ijk, world, pos);
        int prev[3];
        float bx[2], by[2], bz[2];
        float *bases[3] = { bx, by, bz };
        for (int d = 0; d < 3; ++d) {
            prev[d] = (int)floorf(pos[d]);
            float rel = pos[d] - (float)prev[d];
            if (rel < 0) rel = 0;
            bases[d][1] = rel;
            bases[d][0] = 1.f - rel;
        }
        float intensity = 0;
        for (int c = 0; c < 2; ++c) {
            const int Z = prev[2] + c;
            float yv = 0;
            for (int b = 0; b < 2; ++b) {
                const int Y = prev[1] + b;
                float xv = 0;
                for (int a = 0; a < 2; ++a) {
                    const int X = prev[0] + a;
                    const int in = X > -1 && X < fdim[0] && Y > -1 && Y < fdim[1] && Z > -1 && Z < fdim[2];
                    const float v = in ? flo[((size_t)Z * fdim[1] + Y) * fdim[0] + X] : pad;
                    xv += v * bx[a];
                }
                yv += xv * by[b];
            }
            intensity += yv * bz[c];
        }
        warped[i] = intensity;
    }
    return 0;
}

/* The resampling kernels of reg-lib/cpu/_reg_resampling.cpp:60-97, in float with each product
 * and sum rounded on its own (the reference's CPU build has no contraction; this file is ISO C,
 * where gcc contracts nothing either). order 0: nearest (2 taps), 1: linear (2 taps), 3: cubic
 * spline (4 taps starting one voxel before floor(position)). */
static int resample_taps(int order, float rel, float w[4]) {
    if (rel < 0) rel = 0; /* rounding guard of every kernel */
    if (order == 0) {
        w[0] = rel >= 0.5f ? 0.f : 1.f;
        w[1] = rel >= 0.5f ? 1.f : 0.f;
        return 2;
    }
    if (order == 1) {
        w[1] = rel;
        w[0] = 1.f - rel;
        return 2;
    }
    {
        const float sq = rel * rel;
        const float a0 = (2.f - rel) * rel;
        w[0] = (rel * (a0 - 1.f)) / 2.f;
        const float a1 = 3.f * rel - 5.f;
        w[1] = (sq * a1 + 2.f) / 2.f;
        const float a2 = (4.f - 3.f * rel) * rel;
        w[2] = (rel * (a2 + 1.f)) / 2.f;
        w[3] = (rel - 1.f) * sq / 2.f;
        return 4;
    }
}

/* ResampleImage3D with kernel `order` (reg-lib/cpu/_reg_resampling.cpp:316-464): the window of
 * 2 or 4 taps per axis starts at floor(position) - offset; when the whole window lies inside
 * the volume the taps are summed directly, otherwise every out-of-volume tap contributes
 * padding * weight (so NaN padding poisons the voxel even through a zero weight). Sums run x,
 * then y, then z, in float. Masked voxels keep their value. */
int orc_resample_order(const float *flo, const int fdim[3], const float flo_ijk[16], const float *def,
                       const int rdim[3], const int *mask, float pad, int order, float *warped) {
    if (order != 0 && order != 1 && order != 3) return -1;
    const size_t nr = nvox3(rdim);
    const int offset = order == 3 ? 1 : 0;
    for (size_t i = 0; i < nr; ++i) {
        if (mask && mask[i] <= -1) continue;
        const float world[3] = { def[i], def[nr + i], def[2 * nr + i] };
        float pos[3], w[3][4];
        mat44_apply(flo_ijk, world, pos);
        int first[3], n = 0;
        for (int d = 0; d < 3; ++d) {
            const int fl = (int)floorf(pos[d]);
            n = resample_taps(order, pos[d] - (float)fl, w[d]);
            first[d] = fl - offset;
        }
        const int inside = first[0] > -1 && first[0] + n - 1 < fdim[0] && first[1] > -1 &&
                           first[1] + n - 1 < fdim[1] && first[2] > -1 && first[2] + n - 1 < fdim[2];
        float intensity = 0;
        for (int c = 0; c < n; ++c) {
            const int Z = first[2] + c;
            float yv = 0;
            for (int b = 0; b < n; ++b) {
                const int Y = first[1] + b;
                float xv = 0;
                for (int a = 0; a < n; ++a) {
                    const int X = first[0] + a;
                    const int in = inside || (X > -1 && X < fdim[0] && Y > -1 && Y < fdim[1] && Z > -1 && Z < fdim[2]);
                    const float v = in ? flo[((size_t)Z * fdim[1] + Y) * fdim[0] + X] : pad;
                    xv += v * w[0][a];
                }
                yv += xv * w[1][b];
            }
            intensity += yv * w[2][c];
        }
        warped[i] = intensity;
    }
    return 0;
}

/* Spatial gradient of the trilinearly warped floating image in floating-voxel units:
 * TrilinearImageGradient, reg-lib/cpu/_reg_resampling.cpp:1797-1915 (derivative kernel [-1, 1],
 * out-of-volume taps read the padding value, NaN components set to 0, masked voxels get 0). */
int orc_image_gradient_linear(const float *flo, const int fdim[3], const float flo_ijk[16],
                              const float *def, const int rdim[3], const int *mask, float pad,
                              float *grad) {
    const size_t nr = nvox3(rdim);
    const float deriv[2] = { -1.f, 1.f };
    for (size_t i = 0; i < nr; ++i) {
        float g[3] = { 0, 0, 0 };
        if (!mask || mask[i] > -1) {
            const float world[3] = { def[i], def[nr + i], def[2 * nr + i] };
            float pos[3];
            mat44_apply(flo_ijk, world, pos);
            int prev[3];
            float bx[2], by[2], bz[2];
            float *bases[3] = { bx, by, bz };
            for (int d = 0; d < 3; ++d) {
                prev[d] = (int)floorf(pos[d]);
                const float rel = pos[d] - (float)prev[d];
                bases[d][0] = (float)(1.0 - rel);
                bases[d][1] = rel;
            }
            for (int c = 0; c < 2; ++c) {
                const int Z = prev[2] + c;
                const int zin = Z > -1 && Z < fdim[2];
                float xx = 0, yy = 0, zz = 0;
                for (int b = 0; b < 2; ++b) {
                    const int Y = prev[1] + b;
                    const int yzin = zin && Y > -1 && Y < fdim[1];
                    float xt = 0, yt = 0;
                    for (int a = 0; a < 2; ++a) {
                        const int X = prev[0] + a;
                        const float coeff = (yzin && X > -1 && X < fdim[0])
                            ? flo[((size_t)Z * fdim[1] + Y) * fdim[0] + X] : pad;
                        xt += coeff * deriv[a];
                        yt += coeff * bx[a];
                    }
                    xx += xt * by[b];
                    yy += yt * deriv[b];
                    zz += yt * by[b];
                }
                g[0] += xx * bz[c];
                g[1] += yy * bz[c];
                g[2] += zz * deriv[c];
            }
            for (int d = 0; d < 3; ++d)
                if (g[d] != g[d]) g[d] = 0;
        }
        grad[i] = g[0];
        grad[nr + i] = g[1];
        grad[2 * nr + i] = g[2];
    }
    return 0;
}

/* Linear rescale of the finite intensities to [new_min, new_max] in double precision:
 * reg_intensityRescale_core, reg-lib/cpu/_reg_tools.cpp:92-174 (float32 images, slope 1). */
void orc_intensity_rescale(float *img, size_t n, float new_min, float new_max) {
    float mn = FLT_MAX, mx = -FLT_MAX;
    for (size_t i = 0; i < n; ++i) {
        const float v = img[i];
        if (v == v) {
            if (v < mn) mn = v;
            if (v > mx) mx = v;
        }
    }
    const double cur = (double)(mx - mn), nd = (double)(new_max - new_min);
    for (size_t i = 0; i < n; ++i) {
        double v = (double)img[i];
        if (v == v) {
            v = (v - (double)mn) / cur;
            v = v * nd + new_min;
        }
        img[i] = (float)v;
    }
}

/* Cubic B-spline Parzen kernel, reg-lib/cpu/_reg_nmi.h:116-129. The reference writes the
 * constant as the float expression 2.f/3.f even in its double instantiation, so the centre
 * weight is float(2/3) = 0.666666686534881591796875 and the 3-tap smoothing kernel sums to
 * 1 + 2e-8; the histogram total (entropy[3]) carries that factor squared. */
static double parzen(double x) {
    x = x < 0 ? -x : x;
    if (x < 2.0) {
        if (x < 1.0) return (double)(2.0f / 3.0f) + (0.5 * x - 1.0) * x * x;
        x -= 2.0;
        return -x * x * x / 6.0;
    }
    return 0;
}

/* and its derivative, reg-lib/cpu/_reg_nmi.h:131-145 */
static double parzen_deriv(double ox) {
    double x = ox < 0 ? -ox : ox;
    if (x < 2.0) {
        if (x < 1.0) return (1.5 * x - 2.0) * ox;
        x -= 2.0;
        const double v = -0.5 * x * x;
        return ox < 0 ? -v : v;
    }
    return 0;
}

/* NMI with the approximated Parzen window: reg_getNmiValue, reg-lib/cpu/_reg_nmi.cpp:160-347,
 * approximation branch (:214-283) and the ratio of :377-382 with weight 1.
 * Outputs pro/logh (B_r*B_f + B_r + B_f doubles: joint, reference marginal, floating marginal)
 * and ent[4] = {H_ref, H_war, H_joint, total count}. */
double orc_nmi_value(const float *ref, const float *war, size_t n, const int *mask, int rb,
                     int fb, double *pro, double *logh, double *ent) {
    const int total = rb * fb + rb + fb;
    memset(pro, 0, sizeof(double) * total);
    for (size_t i = 0; i < n; ++i) {
        if (mask && mask[i] <= -1) continue;
        const float r = ref[i], w = war[i];
        if (r == r && w == w && 0 <= r && r < rb && 0 <= w && w < fb)
            pro[(int)r + (int)w * rb] += 1.0;
    }
    const double k[3] = { parzen(-1.0), parzen(0.0), parzen(-1.0) };
    memset(logh, 0, sizeof(double) * total);
    for (int f = 0; f < fb; ++f)
        for (int r = 0; r < rb; ++r) {
            double v = 0;
            for (int it = 0; it < 3; ++it) {
                const int idx = r - 1 + it;
                if (-1 < idx && idx < rb) v += pro[idx + rb * f] * k[it];
            }
            logh[r + rb * f] = v;
        }
    for (int r = 0; r < rb; ++r)
        for (int f = 0; f < fb; ++f) {
            double v = 0;
            for (int it = 0; it < 3; ++it) {
                const int idx = f - 1 + it;
                if (-1 < idx && idx < fb) v += logh[r + rb * idx] * k[it];
            }
            pro[r + rb * f] = v;
        }
    double activeVoxel = 0;
    for (int i = 0; i < total; ++i) activeVoxel += pro[i];
    ent[3] = activeVoxel;
    for (int i = 0; i < total; ++i) pro[i] /= activeVoxel;
    for (int r = 0; r < rb; ++r) {
        double s = 0;
        for (int f = 0; f < fb; ++f) s += pro[r + rb * f];
        pro[rb * fb + r] = s;
    }
    for (int f = 0; f < fb; ++f) {
        double s = 0;
        for (int r = 0; r < rb; ++r) s += pro[r + rb * f];
        pro[rb * fb + rb + f] = s;
    }
    memset(logh, 0, sizeof(double) * total);
    double hr = 0, hw = 0, hj = 0;
    for (int r = 0; r < rb; ++r) {
        const double p = pro[rb * fb + r];
        if (p > 0) { const double l = log(p); hr -= p * l; logh[rb * fb + r] = l; }
    }
    for (int f = 0; f < fb; ++f) {
        const double p = pro[rb * fb + rb + f];
        if (p > 0) { const double l = log(p); hw -= p * l; logh[rb * fb + rb + f] = l; }
    }
    for (int i = 0; i < rb * fb; ++i) {
        const double p = pro[i];
        if (p > 0) { const double l = log(p); hj -= p * l; logh[i] = l; }
    }
    ent[0] = hr;
    ent[1] = hw;
    ent[2] = hj;
    return (hr + hw) / hj;
}

/* Voxel-wise NMI gradient added into vgrad: reg_getVoxelBasedNmiGradient3d,
 * reg-lib/cpu/_reg_nmi.cpp:501-593 (FP64 accumulation, 4x4 Parzen window). */
void orc_nmi_voxel_gradient(const float *ref, const float *war, const float *wgrad, size_t n,
                            const int *mask, int rb, int fb, const double *logh,
                            const double *ent, double weight, float *vgrad) {
    const double nmi = (ent[0] + ent[1]) / ent[2];
    const size_t roff = (size_t)rb * fb, foff = roff + rb;
    for (size_t i = 0; i < n; ++i) {
        if (mask && mask[i] <= -1) continue;
        const float r = ref[i], w = war[i];
        if (!(r == r && w == w)) continue;
        const float g[3] = { wgrad[i], wgrad[n + i], wgrad[2 * n + i] };
        double jd[3] = { 0, 0, 0 }, rd[3] = { 0, 0, 0 }, wd[3] = { 0, 0, 0 };
        for (int rr = (int)(r - 1.f); rr < (int)(r + 3.f); ++rr) {
            if (!(-1 < rr && rr < rb)) continue;
            for (int ww = (int)(w - 1.f); ww < (int)(w + 3.f); ++ww) {
                if (!(-1 < ww && ww < fb)) continue;
                const double common = parzen((double)r - rr) * parzen_deriv((double)w - ww);
                const double jl = logh[rr + ww * rb], rl = logh[rr + roff], wl = logh[ww + foff];
                for (int d = 0; d < 3; ++d) {
                    if (g[d] == g[d]) {
                        rd[d] += common * g[d] * rl;
                        wd[d] += common * g[d] * wl;
                        jd[d] += common * g[d] * jl;
                    }
                }
            }
        }
        for (int d = 0; d < 3; ++d)
            vgrad[d * n + i] += (float)(weight * (rd[d] + wd[d] - nmi * jd[d]) / (ent[2] * ent[3]));
    }
}

/* One axis of the density-normalised cubic B-spline convolution:
 * reg_tools_kernelConvolution (Cubic), reg-lib/cpu/_reg_tools.cpp:831-1112 (scalar branch).
 * density = 1 where the mask is >= 0 and the value is finite; the line sums of kernel*value and
 * kernel*density are accumulated in double; result = value/density, NaN where density was 0. */
void orc_kernel_convolution_cubic(float *img, int nvol, const int dim[3], const float pix[3],
                                  float spacing_mm, int axis, const int *mask) {
    const size_t nv = nvox3(dim);
    float *density = (float *)malloc(nv * sizeof(float));
    unsigned char *isnan_ = (unsigned char *)malloc(nv);
    const double tmp = spacing_mm > 0 ? spacing_mm / pix[axis] : fabs(spacing_mm);
    const int radius = (int)(tmp * 2.0f);
    float kernel[4096];
    double ksum = 0;
    for (int i = -radius; i <= radius; ++i) {
        const double rel = fabs(i / tmp);
        float kv;
        if (rel < 1.0) kv = (float)(2.0 / 3.0 - rel * rel + 0.5 * rel * rel * rel);
        else if (rel < 2.0) kv = (float)(-(rel - 2.0) * (rel - 2.0) * (rel - 2.0) / 6.0);
        else kv = 0;
        kernel[i + radius] = kv;
        ksum += kv;
    }
    const int len = dim[axis];
    const size_t stride = axis == 0 ? 1 : axis == 1 ? (size_t)dim[0] : (size_t)dim[0] * dim[1];
    const int planes = axis == 0 ? dim[1] * dim[2] : axis == 1 ? dim[0] * dim[2] : dim[0] * dim[1];
    float *bi = (float *)malloc(sizeof(float) * (len + 1));
    float *bd = (float *)malloc(sizeof(float) * (len + 1));
    for (int t = 0; t < nvol; ++t) {
        float *v = img + (size_t)t * nv;
        for (size_t i = 0; i < nv; ++i) {
            density[i] = ((!mask || mask[i] >= 0) && v[i] == v[i]) ? 1.f : 0.f;
            isnan_[i] = density[i] == 0.f;
            if (isnan_[i]) v[i] = 0;
        }
        if (radius > 0 && dim[axis] > 1 && ksum > 0) {
            for (int p = 0; p < planes; ++p) {
                size_t base;
                if (axis == 0) base = (size_t)p * dim[0];
                else if (axis == 1) base = (size_t)(p / dim[0]) * dim[0] * dim[1] + p % dim[0];
                else base = (size_t)p;
                for (int l = 0; l < len; ++l) {
                    bi[l] = v[base + l * stride];
                    bd[l] = density[base + l * stride];
                }
                for (int l = 0; l < len; ++l) {
                    int pre = l - radius, pst = l + radius + 1;
                    const float *kp = kernel;
                    if (pre < 0) { kp = &kernel[-pre]; pre = 0; }
                    if (pst > len) pst = len;
                    double is = 0, ds = 0;
                    for (int k = pre; k < pst; ++k) {
                        const float kv = *kp++;
                        is += kv * bi[k];
                        ds += kv * bd[k];
                    }
                    v[base + l * stride] = (float)is;
                    density[base + l * stride] = (float)ds;
                }
            }
        }
        for (size_t i = 0; i < nv; ++i)
            v[i] = isnan_[i] ? NAN : v[i] / density[i];
    }
    free(bi);
    free(bd);
    free(density);
    free(isnan_);
}

/* Node gradient from a voxel gradient: reg_voxelCentricToNodeCentric,
 * reg-lib/cpu/_reg_localTrans.cpp:1540-1685 (no affine extension): node -> reference voxel via
 * ref_ijk * grid_xyz, trilinear sample (0 outside), reorientation by the transpose of the 3x3
 * part of `reorient`, weight *= prod_i (row norm i of grid_xyz) / rpix[i]. */
void orc_voxel_to_node(float *node, const int cdim[3], const float grid_xyz[16],
                       const float *voxel, const int rdim[3], const float rpix[3],
                       const float ref_ijk[16], const float reorient[16], float weight,
                       int update) {
    const size_t nc = nvox3(cdim), nr = nvox3(rdim);
    float t[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0;
            for (int k = 0; k < 4; ++k) s += (double)ref_ijk[4 * i + k] * grid_xyz[4 * k + j];
            t[4 * i + j] = (float)s;
        }
    for (int i = 0; i < 3; ++i) {
        const float ratio = sqrtf(grid_xyz[4 * i] * grid_xyz[4 * i] + grid_xyz[4 * i + 1] * grid_xyz[4 * i + 1]
                                  + grid_xyz[4 * i + 2] * grid_xyz[4 * i + 2]);
        weight *= ratio / rpix[i];
    }
    size_t ni = 0;
    for (int z = 0; z < cdim[2]; ++z)
        for (int y = 0; y < cdim[1]; ++y)
            for (int x = 0; x < cdim[0]; ++x, ++ni) {
                const float nc3[3] = { (float)x, (float)y, (float)z };
                float vc[3];
                mat44_apply(t, nc3, vc);
                int pre[3];
                float bx[2], by[2], bz[2];
                float *bases[3] = { bx, by, bz };
                for (int d = 0; d < 3; ++d) {
                    pre[d] = (int)floorf(vc[d]);
                    bases[d][1] = vc[d] - (float)pre[d];
                    bases[d][0] = 1.f - bases[d][1];
                }
                float iv[3] = { 0, 0, 0 };
                for (int c = 0; c < 2; ++c) {
                    const int Z = pre[2] + c;
                    if (Z <= -1 || Z >= rdim[2]) continue;
                    for (int b = 0; b < 2; ++b) {
                        const int Y = pre[1] + b;
                        if (Y <= -1 || Y >= rdim[1]) continue;
                        for (int a = 0; a < 2; ++a) {
                            const int X = pre[0] + a;
                            if (X <= -1 || X >= rdim[0]) continue;
                            const size_t idx = ((size_t)Z * rdim[1] + Y) * rdim[0] + X;
                            const float lw = bx[a] * by[b] * bz[c];
                            iv[0] += lw * voxel[idx];
                            iv[1] += lw * voxel[nr + idx];
                            iv[2] += lw * voxel[2 * nr + idx];
                        }
                    }
                }
                float ro[3];
                for (int d = 0; d < 3; ++d)
                    ro[d] = reorient[0 * 4 + d] * iv[0] + reorient[1 * 4 + d] * iv[1] + reorient[2 * 4 + d] * iv[2];
                for (int d = 0; d < 3; ++d) {
                    if (update) node[d * nc + ni] += ro[d] * weight;
                    else node[d * nc + ni] = ro[d] * weight;
                }
            }
}

/* Compute::ConvolveVoxelBasedMeasureGradient, reg-lib/Compute.cpp:230-281: three one-axis cubic
 * convolutions with the grid spacing (mm), then the node sampling with the floating ijk matrix
 * as reorientation; overwrites node. vgrad is modified in place. */
void orc_convolve_to_nodes(float *vgrad, const int rdim[3], const float rpix[3],
                           const float ref_ijk[16], const int cdim[3], const float cpix[3],
                           const float grid_xyz[16], const float flo_ijk[16], float weight,
                           float *node) {
    orc_kernel_convolution_cubic(vgrad, 3, rdim, rpix, cpix[0], 0, NULL);
    orc_kernel_convolution_cubic(vgrad, 3, rdim, rpix, cpix[1], 1, NULL);
    if (rdim[2] > 1) orc_kernel_convolution_cubic(vgrad, 3, rdim, rpix, cpix[2], 2, NULL);
    orc_voxel_to_node(node, cdim, grid_xyz, vgrad, rdim, rpix, ref_ijk, flo_ijk, weight, 0);
}

/* Second-derivative stencils of the cubic B-spline at the nodes, in the 27-point (c, b, a)
 * order of set_second_order_bspline_basis_values, reg-lib/cpu/_reg_splineBasis.cpp:291-455.
 * The reference tabulates them rounded to 6 decimals; the same rounding is applied here to
 * the exact values B(-1)=B(1)=1/6, B(0)=2/3, B'(-1)=-1/2, B'(0)=0, B'(1)=1/2, B''(+-1)=1,
 * B''(0)=-2. */
static void be_basis(float xx[27], float yy[27], float zz[27], float xy[27], float yz[27], float xz[27]) {
    const double B[3] = { 1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0 };
    const double D[3] = { -0.5, 0.0, 0.5 };
    const double S[3] = { 1.0, -2.0, 1.0 };
    int i = 0;
    for (int c = 0; c < 3; ++c)
        for (int b = 0; b < 3; ++b)
            for (int a = 0; a < 3; ++a, ++i) {
                xx[i] = (float)(round(S[a] * B[b] * B[c] * 1e6) / 1e6);
                yy[i] = (float)(round(B[a] * S[b] * B[c] * 1e6) / 1e6);
                zz[i] = (float)(round(B[a] * B[b] * S[c] * 1e6) / 1e6);
                xy[i] = (float)(round(D[a] * D[b] * B[c] * 1e6) / 1e6);
                yz[i] = (float)(round(B[a] * D[b] * D[c] * 1e6) / 1e6);
                xz[i] = (float)(round(D[a] * B[b] * D[c] * 1e6) / 1e6);
            }
}

/* Approximate bending energy on the interior nodes, computed on the positions:
 * reg_spline_approxBendingEnergyValue3D, reg-lib/cpu/_reg_localTrans_regul.cpp:72-153
 * (sum in double, divided by the number of grid values, 3 per node). */
double orc_be_value(const float *cpp, const int cdim[3]) {
    const size_t nc = nvox3(cdim);
    float bxx[27], byy[27], bzz[27], bxy[27], byz[27], bxz[27];
    be_basis(bxx, byy, bzz, bxy, byz, bxz);
    double total = 0;
    for (int z = 1; z < cdim[2] - 1; ++z)
        for (int y = 1; y < cdim[1] - 1; ++y)
            for (int x = 1; x < cdim[0] - 1; ++x) {
                float d[3][6] = { { 0 } };
                int i = 0;
                for (int c = -1; c < 2; ++c)
                    for (int b = -1; b < 2; ++b)
                        for (int a = -1; a < 2; ++a, ++i) {
                            const size_t idx = ((size_t)(z + c) * cdim[1] + y + b) * cdim[0] + x + a;
                            for (int k = 0; k < 3; ++k) {
                                const float v = cpp[k * nc + idx];
                                d[k][0] += bxx[i] * v;
                                d[k][1] += byy[i] * v;
                                d[k][2] += bzz[i] * v;
                                d[k][3] += bxy[i] * v;
                                d[k][4] += byz[i] * v;
                                d[k][5] += bxz[i] * v;
                            }
                        }
                /* evaluation order of the reference expression: the first three squares sum in
                 * float, everything after the first 2.0* term accumulates in double */
                double s = (double)(d[0][0] * d[0][0] + d[0][1] * d[0][1] + d[0][2] * d[0][2])
                           + 2.0 * (double)(d[0][3] * d[0][3] + d[0][4] * d[0][4] + d[0][5] * d[0][5]);
                for (int k = 1; k < 3; ++k) {
                    s += (double)(d[k][0] * d[k][0]);
                    s += (double)(d[k][1] * d[k][1]);
                    s += (double)(d[k][2] * d[k][2]);
                    s += 2.0 * (double)(d[k][3] * d[k][3] + d[k][4] * d[k][4] + d[k][5] * d[k][5]);
                }
                total += s;
            }
    return total / (double)(3 * nc);
}

/* Bending-energy gradient added into grad: reg_spline_approxBendingEnergyGradient3D,
 * reg-lib/cpu/_reg_localTrans_regul.cpp:286-451. Works on displacements (position minus the
 * node's own position grid_xyz*(x,y,z), :311 and _reg_tools.cpp:1988-2032), zero outside the
 * grid, 18 derivative values per node (cross terms doubled), then the stencil applied again
 * with basis[a] at neighbour offset a; grad += weight/#nodes * sum. */
void orc_be_gradient(const float *cpp, const int cdim[3], const float grid_xyz[16], float weight,
                     float *grad) {
    const size_t nc = nvox3(cdim);
    float bxx[27], byy[27], bzz[27], bxy[27], byz[27], bxz[27];
    be_basis(bxx, byy, bzz, bxy, byz, bxz);
    float *disp = (float *)malloc(3 * nc * sizeof(float));
    float *der = (float *)calloc(18 * nc, sizeof(float));
    size_t idx = 0;
    for (int z = 0; z < cdim[2]; ++z)
        for (int y = 0; y < cdim[1]; ++y)
            for (int x = 0; x < cdim[0]; ++x, ++idx)
                for (int k = 0; k < 3; ++k) {
                    const float init = grid_xyz[4 * k] * (float)x + grid_xyz[4 * k + 1] * (float)y
                                       + grid_xyz[4 * k + 2] * (float)z + grid_xyz[4 * k + 3];
                    disp[k * nc + idx] = cpp[k * nc + idx] - init;
                }
    idx = 0;
    for (int z = 0; z < cdim[2]; ++z)
        for (int y = 0; y < cdim[1]; ++y)
            for (int x = 0; x < cdim[0]; ++x, ++idx) {
                float d[3][6] = { { 0 } };
                int i = 0;
                for (int c = -1; c < 2; ++c)
                    for (int b = -1; b < 2; ++b)
                        for (int a = -1; a < 2; ++a, ++i) {
                            const int X = x + a, Y = y + b, Z = z + c;
                            if (X < 0 || Y < 0 || Z < 0 || X >= cdim[0] || Y >= cdim[1] || Z >= cdim[2]) continue;
                            const size_t j = ((size_t)Z * cdim[1] + Y) * cdim[0] + X;
                            for (int k = 0; k < 3; ++k) {
                                const float v = disp[k * nc + j];
                                d[k][0] += bxx[i] * v;
                                d[k][1] += byy[i] * v;
                                d[k][2] += bzz[i] * v;
                                d[k][3] += bxy[i] * v;
                                d[k][4] += byz[i] * v;
                                d[k][5] += bxz[i] * v;
                            }
                        }
                float *o = der + 18 * idx;
                for (int t = 0; t < 3; ++t)
                    for (int k = 0; k < 3; ++k)
                        o[3 * t + k] = d[k][t];
                for (int t = 3; t < 6; ++t)
                    for (int k = 0; k < 3; ++k)
                        o[3 * t + k] = (float)(2.0 * d[k][t]);
            }
    const float ratio = weight / (float)nc;
    const float *bases[6] = { bxx, byy, bzz, bxy, byz, bxz };
    idx = 0;
    for (int z = 0; z < cdim[2]; ++z)
        for (int y = 0; y < cdim[1]; ++y)
            for (int x = 0; x < cdim[0]; ++x, ++idx) {
                float g[3] = { 0, 0, 0 };
                int a = 0;
                for (int Z = z - 1; Z < z + 2; ++Z)
                    for (int Y = y - 1; Y < y + 2; ++Y)
                        for (int X = x - 1; X < x + 2; ++X, ++a) {
                            if (X < 0 || Y < 0 || Z < 0 || X >= cdim[0] || Y >= cdim[1] || Z >= cdim[2]) continue;
                            const float *p = der + 18 * (((size_t)Z * cdim[1] + Y) * cdim[0] + X);
                            for (int t = 0; t < 6; ++t)
                                for (int k = 0; k < 3; ++k) g[k] += p[3 * t + k] * bases[t][a];
                        }
                for (int k = 0; k < 3; ++k) grad[k * nc + idx] += ratio * g[k];
            }
    free(disp);
    free(der);
}

/* Largest node-gradient length in float: reg_getMaximalLength, reg-lib/cpu/_reg_tools.cpp:335-371 */
double orc_max_length(const float *grad, size_t nnode, int ox, int oy, int oz) {
    float mx = 0;
    for (size_t i = 0; i < nnode; ++i) {
        const float x = ox ? grad[i] : 0, y = oy ? grad[nnode + i] : 0, z = oz ? grad[2 * nnode + i] : 0;
        const float l = (float)sqrt(x * x + y * y + z * z);
        if (l > mx) mx = l;
    }
    return mx;
}

/* Compute::NormaliseGradient, reg-lib/Compute.cpp:148-176 */
void orc_normalise_gradient(float *grad, size_t nnode, double maxlen, int ox, int oy, int oz) {
    if (maxlen == 0 || (!ox && !oy && !oz)) return;
    const double inv = 1.0 / maxlen;
    for (size_t i = 0; i < nnode; ++i) {
        const double x = ox ? (double)grad[i] : 0, y = oy ? (double)grad[nnode + i] : 0,
                     z = oz ? (double)grad[2 * nnode + i] : 0;
        grad[i] = (float)(x * inv);
        grad[nnode + i] = (float)(y * inv);
        grad[2 * nnode + i] = (float)(z * inv);
    }
}

/* Compute::UpdateControlPointPosition, reg-lib/Compute.cpp:91-107 (all axes optimised) */
void orc_update_control_points(float *cur, const float *best, const float *grad, float scale,
                               size_t nvox) {
    for (size_t i = 0; i < nvox; ++i) cur[i] = best[i] + scale * grad[i];
}

/* ConjugateGradient::UpdateGradientValues, reg-lib/Optimiser.cpp:231-317 (forward only):
 * first call g1 = g2 = -grad; later gam = sum((grad+g1)*grad) / sum(g2*g1) in double,
 * g1 = -grad, g2 = g1 + gam*g2, grad = -g2. */
void orc_cg_update(float *grad, float *g1, float *g2, size_t nvox, int first_call) {
    if (first_call) {
        for (size_t i = 0; i < nvox; ++i) g2[i] = g1[i] = -grad[i];
        return;
    }
    double dgg = 0, gg = 0;
    for (size_t i = 0; i < nvox; ++i) {
        gg += g2[i] * g1[i];
        dgg += (grad[i] + g1[i]) * grad[i];
    }
    const double gam = dgg / gg;
    for (size_t i = 0; i < nvox; ++i) {
        g1[i] = -grad[i];
        g2[i] = (float)(g1[i] + gam * g2[i]);
        grad[i] = -g2[i];
    }
}
