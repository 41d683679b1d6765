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

/* ------------------------------------------------------------------------------------------
 * F3D2 (reg_f3d2): velocity fields
 * ------------------------------------------------------------------------------------------ */

/* the affine inverse of nifti_mat44_inverse (reg-io/niftilib): the 3x3 block by cofactors over
 * the determinant in double, the translation as -inverse * t, rounded to float */
static void mat44_inverse(const float m[16], float out[16]) {
    const double r11 = m[0], r12 = m[1], r13 = m[2], r21 = m[4], r22 = m[5], r23 = m[6];
    const double r31 = m[8], r32 = m[9], r33 = m[10], v1 = m[3], v2 = m[7], v3 = m[11];
    double deti = r11 * r22 * r33 - r11 * r32 * r23 - r21 * r12 * r33 + r21 * r32 * r13 + r31 * r12 * r23 -
                  r31 * r22 * r13;
    if (deti != 0.0) deti = 1.0 / deti;
    out[0] = (float)(deti * (r22 * r33 - r32 * r23));
    out[1] = (float)(deti * (-r12 * r33 + r32 * r13));
    out[2] = (float)(deti * (r12 * r23 - r22 * r13));
    out[3] = (float)(deti * (-r12 * r23 * v3 + r12 * v2 * r33 + r22 * r13 * v3 - r22 * v1 * r33 - r32 * r13 * v2 +
                             r32 * v1 * r23));
    out[4] = (float)(deti * (-r21 * r33 + r31 * r23));
    out[5] = (float)(deti * (r11 * r33 - r31 * r13));
    out[6] = (float)(deti * (-r11 * r23 + r21 * r13));
    out[7] = (float)(deti * (r11 * r23 * v3 - r11 * v2 * r33 - r21 * r13 * v3 + r21 * v1 * r33 + r31 * r13 * v2 -
                             r31 * v1 * r23));
    out[8] = (float)(deti * (r21 * r32 - r31 * r22));
    out[9] = (float)(deti * (-r11 * r32 + r31 * r12));
    out[10] = (float)(deti * (r11 * r22 - r21 * r12));
    out[11] = (float)(deti * (-r11 * r22 * v3 + r11 * r32 * v2 + r21 * r12 * v3 - r21 * r32 * v1 - r31 * r12 * v2 +
                              r31 * r22 * v1));
    out[12] = out[13] = out[14] = 0.f;
    out[15] = (float)(deti != 0.0 ? 1.0 : 0.0);
}

/* m[r][0] * x + m[r][1] * y + m[r][2] * z + m[r][3] in float, left to right: the conversions of
 * reg_getDeformationFromDisplacement_3D (reg-lib/cpu/_reg_tools.cpp:2107-2150) and of the
 * composition paths (reg-lib/cpu/_reg_localTrans.cpp:925-940, 2380-2395) */
static float row_f(const float *m, float x, float y, float z) {
    float v = m[0] * x;
    v = v + m[1] * y;
    v = v + m[2] * z;
    return v + m[3];
}

/* get_SlidedValues for positions (reg-lib/cpu/_reg_splineBasis.cpp:497-550) */
static void slided3(const float *px, const float *py, const float *pz, int x, int y, int z, const int d[3],
                    const float xyz[16], float *vx, float *vy, float *vz) {
    const int nx = x < 0 ? 0 : (x >= d[0] ? d[0] - 1 : x);
    const int ny = y < 0 ? 0 : (y >= d[1] ? d[1] - 1 : y);
    const int nz = z < 0 ? 0 : (z >= d[2] ? d[2] - 1 : z);
    const int sx = x - nx, sy = y - ny, sz = z - nz;
    const float shx = (float)sx * xyz[0] + (float)sy * xyz[1] + (float)sz * xyz[2];
    const float shy = (float)sx * xyz[4] + (float)sy * xyz[5] + (float)sz * xyz[6];
    const float shz = (float)sx * xyz[8] + (float)sy * xyz[9] + (float)sz * xyz[10];
    const size_t i = ((size_t)nz * d[1] + ny) * d[0] + nx;
    *vx = px[i] + shx;
    *vy = py[i] + shy;
    *vz = pz[i] + shz;
}

/* the flow of a velocity grid at every voxel of a field, as a displacement (mm): the identity
 * positions of reg_spline_getFlowFieldFromVelocityGrid (:3465-3491) through the composition
 * branch of reg_cubic_spline_getDeformationField3D with the SSE build's sums (:903-1079: four
 * x-lanes accumulated over (z, y), then added in lane order; the grid values of get_GridValues,
 * reg-lib/cpu/_reg_splineBasis.cpp:603-663, whose rows after an outside one take the sliding
 * path), then reg_getDisplacementFromDeformation. Also the extrema of all components. */
static void velocity_flow(const float *vel, const int gdim[3], const float gxyz[16], const float gijk[16],
                          const int fdim[3], const float fxyz[16], float *disp, float *lo, float *hi) {
    const size_t n = nvox3(fdim), gn = nvox3(gdim);
    const float *cx = vel, *cy = vel + gn, *cz = vel + 2 * gn;
    *lo = FLT_MAX;
    *hi = -FLT_MAX;
    for (int z = 0; z < fdim[2]; ++z)
        for (int y = 0; y < fdim[1]; ++y)
            for (int x = 0; x < fdim[0]; ++x) {
                const size_t i = ((size_t)z * fdim[1] + y) * fdim[0] + x;
                const float rx = row_f(fxyz, (float)x, (float)y, (float)z);
                const float ry = row_f(fxyz + 4, (float)x, (float)y, (float)z);
                const float rz = row_f(fxyz + 8, (float)x, (float)y, (float)z);
                const float v[3] = { row_f(gijk, rx, ry, rz), row_f(gijk + 4, rx, ry, rz), row_f(gijk + 8, rx, ry, rz) };
                int pre[3];
                float bas[3][4];
                for (int k = 0; k < 3; ++k) {
                    pre[k] = (int)floorf(v[k]);
                    float b = v[k] - (float)pre[k];
                    pre[k] -= 1;
                    if (b < 0) b = 0;
                    orc_bspline_basis(b, bas[k]);
                }
                float gx[64], gy[64], gz[64];
                int coord = 0;
                for (int Z = pre[2]; Z < pre[2] + 4; ++Z) {
                    int out = !(Z > -1 && Z < gdim[2]);
                    for (int Y = pre[1]; Y < pre[1] + 4; ++Y) {
                        if (!(Y > -1 && Y < gdim[1])) out = 1;
                        for (int X = pre[0]; X < pre[0] + 4; ++X, ++coord) {
                            if (X > -1 && X < gdim[0] && !out) {
                                const size_t j = ((size_t)Z * gdim[1] + Y) * gdim[0] + X;
                                gx[coord] = cx[j];
                                gy[coord] = cy[j];
                                gz[coord] = cz[j];
                            } else {
                                slided3(cx, cy, cz, X, Y, Z, gdim, gxyz, &gx[coord], &gy[coord], &gz[coord]);
                            }
                        }
                    }
                }
                float tx[4] = { 0, 0, 0, 0 }, ty[4] = { 0, 0, 0, 0 }, tz[4] = { 0, 0, 0, 0 };
                for (int c = 0; c < 4; ++c)
                    for (int b = 0; b < 4; ++b) {
                        const float yz = bas[1][b] * bas[2][c];
                        for (int a = 0; a < 4; ++a) {
                            const float w = yz * bas[0][a];
                            tx[a] = w * gx[c * 16 + b * 4 + a] + tx[a];
                            ty[a] = w * gy[c * 16 + b * 4 + a] + ty[a];
                            tz[a] = w * gz[c * 16 + b * 4 + a] + tz[a];
                        }
                    }
                const float d[3] = { tx[0] + tx[1] + tx[2] + tx[3] - rx, ty[0] + ty[1] + ty[2] + ty[3] - ry,
                                     tz[0] + tz[1] + tz[2] + tz[3] - rz };
                for (int k = 0; k < 3; ++k) {
                    disp[k * n + i] = d[k];
                    if (d[k] < *lo) *lo = d[k];
                    if (d[k] > *hi) *hi = d[k];
                }
            }
}

/* reg_defField_compose3D (reg-lib/cpu/_reg_localTrans.cpp:2334-2458): upd(x) <- app(upd(x)) */
static void compose3(const float *app, float *upd, const int dim[3], const float xyz[16], const float ijk[16]) {
    const size_t n = nvox3(dim);
    const float *ax = app, *ay = app + n, *az = app + 2 * n;
    for (size_t i = 0; i < n; ++i) {
        const float p0 = upd[i], p1 = upd[n + i], p2 = upd[2 * n + i];
        const float v[3] = { row_f(ijk, p0, p1, p2), row_f(ijk + 4, p0, p1, p2), row_f(ijk + 8, p0, p1, p2) };
        int pre[3];
        float rel[3][2];
        for (int k = 0; k < 3; ++k) {
            pre[k] = (int)floorf(v[k]);
            rel[k][1] = v[k] - (float)pre[k];
            rel[k][0] = 1.f - rel[k][1];
        }
        float r0 = 0, r1 = 0, r2 = 0;
        for (int c = 0; c < 2; ++c) {
            const int Z = pre[2] + c;
            const int inZ = Z > -1 && Z < dim[2];
            for (int b = 0; b < 2; ++b) {
                const int Y = pre[1] + b;
                const float tb = rel[1][b] * rel[2][c];
                const int inY = Y > -1 && Y < dim[1];
                for (int a = 0; a < 2; ++a) {
                    const int X = pre[0] + a;
                    float dx, dy, dz;
                    if (X > -1 && X < dim[0] && inY && inZ) {
                        const size_t j = ((size_t)Z * dim[1] + Y) * dim[0] + X;
                        dx = ax[j];
                        dy = ay[j];
                        dz = az[j];
                    } else {
                        slided3(ax, ay, az, X, Y, Z, dim, xyz, &dx, &dy, &dz);
                    }
                    const float w = rel[0][a] * tb;
                    r0 += dx * w;
                    r1 += dy * w;
                    r2 += dz * w;
                }
            }
        }
        upd[i] = r0;
        upd[n + i] = r1;
        upd[2 * n + i] = r2;
    }
}

int orc_velocity_squaring_steps(float lo, float hi) {
    float extrema = fabsf(lo) > hi ? fabsf(lo) : hi;
    int steps = 1;
    while (extrema / (float)pow(2, steps) >= 0.28f) ++steps;
    return steps > 6 ? steps : 6;
}

/* the flow divided by 2^N (reg_tools_divideValueToImage: in double, rounded to float) and turned
 * back into positions */
static void flow_scale(float *d, const int dim[3], const float xyz[16], int steps) {
    const size_t n = nvox3(dim);
    const double s = (double)(float)pow(2, steps);
    for (int z = 0; z < dim[2]; ++z)
        for (int y = 0; y < dim[1]; ++y)
            for (int x = 0; x < dim[0]; ++x) {
                const size_t i = ((size_t)z * dim[1] + y) * dim[0] + x;
                for (int k = 0; k < 3; ++k)
                    d[k * n + i] = (float)((double)d[k * n + i] / s) + row_f(xyz + 4 * k, (float)x, (float)y, (float)z);
            }
}

/* reg_spline_getDefFieldFromVelocityGrid (reg-lib/cpu/_reg_localTrans.cpp:3583-3613) with
 * reg_defField_getDeformationFieldFromFlowField (:3494-3580), no affine: N = steps, recomputed
 * from the flow's extrema when update (or steps == 0); the scaled flow squared N times. */
int orc_velocity_def_field(const float *vel, const int gdim[3], const float gxyz[16], int steps, int update,
                           const int fdim[3], const float fxyz[16], float *def, int *steps_out) {
    const size_t n = nvox3(fdim);
    float gijk[16], fijk[16], lo, hi;
    mat44_inverse(gxyz, gijk);
    mat44_inverse(fxyz, fijk);
    velocity_flow(vel, gdim, gxyz, gijk, fdim, fxyz, def, &lo, &hi);
    if (update || steps == 0) steps = orc_velocity_squaring_steps(lo, hi);
    flow_scale(def, fdim, fxyz, steps);
    float *tmp = (float *)malloc(3 * n * sizeof(float));
    if (!tmp) return -1;
    for (int k = 0; k < steps; ++k) {
        memcpy(tmp, def, 3 * n * sizeof(float));
        compose3(tmp, def, fdim, fxyz, fijk);
    }
    free(tmp);
    *steps_out = steps;
    return 0;
}

void orc_def_compose(const int dim[3], const float xyz[16], const float *apply, float *update) {
    float ijk[16];
    mat44_inverse(xyz, ijk);
    compose3(apply, update, dim, xyz, ijk);
}

/* the orthogonal factor of a 3x3 matrix (nifti_mat33_polar's role), scaled Newton iteration in
 * double; exactly the identity for a diagonal matrix with positive entries */
static void polar3(const double A[3][3], double Q[3][3]) {
    double X[3][3];
    memcpy(X, A, sizeof(X));
    for (int it = 0; it < 100; ++it) {
        const double det = X[0][0] * (X[1][1] * X[2][2] - X[1][2] * X[2][1]) -
                           X[0][1] * (X[1][0] * X[2][2] - X[1][2] * X[2][0]) +
                           X[0][2] * (X[1][0] * X[2][1] - X[1][1] * X[2][0]);
        if (det == 0.0) break;
        double Y[3][3];
        Y[0][0] = (X[1][1] * X[2][2] - X[1][2] * X[2][1]) / det;
        Y[0][1] = (X[1][2] * X[2][0] - X[1][0] * X[2][2]) / det;
        Y[0][2] = (X[1][0] * X[2][1] - X[1][1] * X[2][0]) / det;
        Y[1][0] = (X[0][2] * X[2][1] - X[0][1] * X[2][2]) / det;
        Y[1][1] = (X[0][0] * X[2][2] - X[0][2] * X[2][0]) / det;
        Y[1][2] = (X[0][1] * X[2][0] - X[0][0] * X[2][1]) / det;
        Y[2][0] = (X[0][1] * X[1][2] - X[0][2] * X[1][1]) / det;
        Y[2][1] = (X[0][2] * X[1][0] - X[0][0] * X[1][2]) / det;
        Y[2][2] = (X[0][0] * X[1][1] - X[0][1] * X[1][0]) / det;
        double nx = 0, ny = 0, dif = 0;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                nx += X[r][c] * X[r][c];
                ny += Y[r][c] * Y[r][c];
            }
        const double g = sqrt(sqrt(ny / nx));
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                const double v = 0.5 * (g * X[r][c] + Y[r][c] / g);
                dif += fabs(v - X[r][c]);
                X[r][c] = v;
            }
        if (dif < 1e-15) break;
    }
    memcpy(Q, X, sizeof(X));
}

/* reg_trilinearResampleGradient (reg-lib/cpu/_reg_resampling.cpp:1537-1766) with padding 0, the
 * gradient image and the field on one grid (dim, xyz, ijk): trilinear sample of g at def(x),
 * times the finite-difference Jacobian of def (the reference's 8-term weight loop, backward at
 * the last index) premultiplied by `reorient` and divided by the real spacing per column */
static void resample_gradient(const float *g, float *out, const float *def, const int dim[3], const float ijk[16],
                              const float R[9], const float sp[3]) {
    const size_t n = nvox3(dim);
    const float *gx = g, *gy = g + n, *gz = g + 2 * n;
    const float *dx = def, *dy = def + n, *dz = def + 2 * n;
    const float basis[2] = { 1.f, 0.f }, deriv[2] = { -1.f, 1.f };
    for (int z = 0; z < dim[2]; ++z)
        for (int y = 0; y < dim[1]; ++y)
            for (int x = 0; x < dim[0]; ++x) {
                const size_t i = ((size_t)z * dim[1] + y) * dim[0] + x;
                const float D0 = dx[i], D1 = dy[i], D2 = dz[i];
                const float c[3] = { row_f(ijk, D0, D1, D2), row_f(ijk + 4, D0, D1, D2), row_f(ijk + 8, D0, D1, D2) };
                int lo[3][2];
                float bw[3][2];
                for (int k = 0; k < 3; ++k) {
                    lo[k][0] = (int)floorf(c[k]);
                    lo[k][1] = (int)ceilf(c[k]);
                    bw[k][1] = fabsf(c[k] - (float)lo[k][0]);
                    bw[k][0] = 1.f - bw[k][1];
                }
                float vx = 0, vy = 0, vz = 0;
                for (int cc = 0; cc < 2; ++cc) {
                    if (lo[2][cc] > -1 && lo[2][cc] < dim[2]) {
                        for (int b = 0; b < 2; ++b) {
                            if (lo[1][b] > -1 && lo[1][b] < dim[1]) {
                                for (int a = 0; a < 2; ++a) {
                                    const float w = bw[0][a] * bw[1][b] * bw[2][cc];
                                    if (lo[0][a] > -1 && lo[0][a] < dim[0]) {
                                        const size_t j = ((size_t)lo[2][cc] * dim[1] + lo[1][b]) * dim[0] + lo[0][a];
                                        vx += gx[j] * w;
                                        vy += gy[j] * w;
                                        vz += gz[j] * w;
                                    } else {
                                        vx += 0.f * w;
                                        vy += 0.f * w;
                                        vz += 0.f * w;
                                    }
                                }
                            } else {
                                vx += 0.f * bw[1][b] * bw[2][cc];
                                vy += 0.f * bw[1][b] * bw[2][cc];
                                vz += 0.f * bw[1][b] * bw[2][cc];
                            }
                        }
                    } else {
                        vx += 0.f * bw[2][cc];
                        vy += 0.f * bw[2][cc];
                        vz += 0.f * bw[2][cc];
                    }
                }
                float J[3][3] = { { 0, 0, 0 }, { 0, 0, 0 }, { 0, 0, 0 } };
                for (int cc = 0; cc < 2; ++cc) {
                    int Z = z + cc;
                    float bz0 = basis[cc], bz1 = deriv[cc];
                    if (z == dim[2] - 1) {
                        if (cc == 1) Z -= 2;
                        bz0 = fabsf(bz0 - 1);
                        bz1 *= -1;
                    }
                    for (int b = 0; b < 2; ++b) {
                        int Y = y + b;
                        float by0 = basis[b], by1 = deriv[b];
                        if (y == dim[1] - 1) {
                            if (b == 1) Y -= 2;
                            by0 = fabsf(by0 - 1);
                            by1 *= -1;
                        }
                        for (int a = 0; a < 2; ++a) {
                            int X = x + a;
                            float bx0 = basis[a], bx1 = deriv[a];
                            if (x == dim[0] - 1) {
                                if (a == 1) X -= 2;
                                bx0 = fabsf(bx0 - 1);
                                bx1 *= -1;
                            }
                            const float w0 = bx1 * by0 * bz0, w1 = bx0 * by1 * bz0, w2 = bx0 * by0 * bz1;
                            const size_t j = ((size_t)Z * dim[1] + Y) * dim[0] + X;
                            const float e[3] = { dx[j], dy[j], dz[j] };
                            for (int r = 0; r < 3; ++r) {
                                J[r][0] += w0 * e[r];
                                J[r][1] += w1 * e[r];
                                J[r][2] += w2 * e[r];
                            }
                        }
                    }
                }
                float M[3][3];
                for (int r = 0; r < 3; ++r)
                    for (int col = 0; col < 3; ++col)
                        M[r][col] = R[3 * r] * J[0][col] + R[3 * r + 1] * J[1][col] + R[3 * r + 2] * J[2][col];
                for (int r = 0; r < 3; ++r)
                    for (int col = 0; col < 3; ++col) M[r][col] /= sp[col];
                out[i] = M[0][0] * vx + M[0][1] * vy + M[0][2] * vz;
                out[n + i] = M[1][0] * vx + M[1][1] * vy + M[1][2] * vz;
                out[2 * n + i] = M[2][0] * vx + M[2][1] * vy + M[2][2] * vz;
            }
}

/* Compute::ExponentiateGradient (reg-lib/Compute.cpp:288-330, no affine): the opposite velocity
 * grid's intermediate fields on the gradient's grid (reg_spline_getIntermediateDefFieldFromVelGrid,
 * reg-lib/cpu/_reg_localTrans.cpp:3616-3681), then for each of them the gradient resampled
 * (reg_resampleGradient, linear, padding 0) and added, then the division by 2^N */
int orc_exponentiate_gradient(const int fdim[3], const float fxyz[16], const float *vel, const int gdim[3],
                              const float gxyz[16], int steps, float *vgrad) {
    const size_t n = nvox3(fdim);
    float gijk[16], fijk[16], lo, hi;
    mat44_inverse(gxyz, gijk);
    mat44_inverse(fxyz, fijk);
    float *fields = (float *)malloc((size_t)steps * 3 * n * sizeof(float));
    float *tmp = (float *)malloc(3 * n * sizeof(float));
    if (!fields || !tmp) {
        free(fields);
        free(tmp);
        return -1;
    }
    velocity_flow(vel, gdim, gxyz, gijk, fdim, fxyz, fields, &lo, &hi);
    flow_scale(fields, fdim, fxyz, steps);
    for (int k = 1; k < steps; ++k) {
        memcpy(fields + (size_t)k * 3 * n, fields + (size_t)(k - 1) * 3 * n, 3 * n * sizeof(float));
        compose3(fields + (size_t)(k - 1) * 3 * n, fields + (size_t)k * 3 * n, fdim, fxyz, fijk);
    }
    double A[3][3], Q[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) A[r][c] = fxyz[4 * r + c];
    polar3(A, Q);
    float R[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) R[3 * r + c] = (float)Q[c][r];
    float sp[3];
    {
        const float o[3] = { 0, 0, 0 };
        float p0[3];
        mat44_apply(fxyz, o, p0);
        for (int c = 0; c < 3; ++c) {
            float e[3] = { 0, 0, 0 }, p1[3];
            e[c] = 1;
            mat44_apply(fxyz, e, p1);
            const float a = p0[0] - p1[0], b = p0[1] - p1[1], d = p0[2] - p1[2];
            sp[c] = sqrtf(a * a + b * b + d * d);
        }
    }
    for (int k = 0; k < steps; ++k) {
        resample_gradient(vgrad, tmp, fields + (size_t)k * 3 * n, fdim, fijk, R, sp);
        for (size_t i = 0; i < 3 * n; ++i) vgrad[i] = (float)((double)tmp[i] + (double)vgrad[i]);
    }
    const double s = pow(2, steps);
    for (size_t i = 0; i < 3 * n; ++i) vgrad[i] = (float)((double)vgrad[i] / s);
    free(fields);
    free(tmp);
    return 0;
}

/* Compute::SymmetriseVelocityFields (reg-lib/Compute.cpp:356-392) */
void orc_symmetrise(const int gdim[3], const float fw_xyz[16], const float bw_xyz[16], float *fw, float *bw) {
    const size_t n = nvox3(gdim);
    for (int z = 0; z < gdim[2]; ++z)
        for (int y = 0; y < gdim[1]; ++y)
            for (int x = 0; x < gdim[0]; ++x) {
                const size_t i = ((size_t)z * gdim[1] + y) * gdim[0] + x;
                for (int k = 0; k < 3; ++k) {
                    const float idf = row_f(fw_xyz + 4 * k, (float)x, (float)y, (float)z);
                    const float idb = row_f(bw_xyz + 4 * k, (float)x, (float)y, (float)z);
                    const float df = fw[k * n + i] - idf, db = bw[k * n + i] - idb;
                    fw[k * n + i] = (float)((double)(df - db) * 0.5) + idf;
                    bw[k * n + i] = (float)((double)(db - df) * 0.5) + idb;
                }
            }
}
