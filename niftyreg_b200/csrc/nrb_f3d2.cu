// F3D2 (reg_f3d2, reg-lib/_reg_f3d2.cpp) on the device: the stationary velocity field of a
// cubic B-spline grid exponentiated by scaling and squaring, composition of deformation fields,
// the "Dartel-like" gradient exponentiation and the symmetrisation of the forward and backward
// velocity grids.
//
// This file is compiled with -fmad=false: every float expression below rounds each product and
// each sum on its own, in the order written, which is the reference's (its SSE build has no
// fused multiply-add), so the arithmetic is the reference's and not a contraction of it.
//
// Every kernel is one thread per voxel (or node) and streams its vector fields through HBM
// (planar x | y | z layout, the NIfTI vector layout); the gathers of the composition and the
// gradient resampling hit L1/L2 because neighbouring threads read neighbouring voxels.

#include <cmath>
#include <cstring>
#include <vector>

#include "nrb_common.cuh"

namespace nrb {

namespace {

// a dense field over an image grid: dims, voxel -> mm and mm -> voxel (first three rows)
struct FieldGeom {
    int nx, ny, nz;
    Mat34 xyz, ijk;
};

FieldGeom field_geom(const int32_t dim[3], const float xyz[16], const float ijk[16]) {
    FieldGeom f;
    f.nx = dim[0];
    f.ny = dim[1];
    f.nz = dim[2];
    f.xyz = to_mat34(xyz);
    f.ijk = to_mat34(ijk);
    return f;
}

// m0 * x + m1 * y + m2 * z + m3, left to right: the voxel -> mm conversions of
// reg_getDeformationFromDisplacement (reg-lib/cpu/_reg_tools.cpp:2107-2150) and the mm -> voxel
// conversions of the composition (reg-lib/cpu/_reg_localTrans.cpp:2380-2395)
__device__ __forceinline__ float row(const float *m, float x, float y, float z) {
    return m[0] * x + m[1] * y + m[2] * z + m[3];
}

__device__ __forceinline__ int floor_int(float v) {
    // Floor<int> of the reference, clamped so that a position far outside (or NaN) stays a
    // defined integer; the sliding clamp below keeps every read inside the field
    float f = floorf(v);
    f = f != f ? 0.f : fminf(fmaxf(f, -1073741824.f), 1073741824.f);
    return (int)f;
}
__device__ __forceinline__ int ceil_int(float v) {
    float f = ceilf(v);
    f = f != f ? 0.f : fminf(fmaxf(f, -1073741824.f), 1073741824.f);
    return (int)f;
}

// get_BSplineBasisValues (reg-lib/cpu/_reg_splineBasis.cpp:17-26): the cube and the polynomial
// sums in double, as the reference writes them
__device__ __forceinline__ void bspline_basis_f64(float b, float v[4]) {
    const float ff = b * b, fff = ff * b;
    const float mf = (float)(1.0 - (double)b);
    v[0] = (float)((double)(mf * mf * mf) / 6.0);
    v[1] = (float)((3.0 * (double)fff - 6.0 * (double)ff + 4.0) / 6.0);
    v[2] = (float)((-3.0 * (double)fff + 3.0 * (double)ff + 3.0 * (double)b + 1.0) / 6.0);
    v[3] = (float)((double)fff / 6.0);
}

// get_SlidedValues (reg-lib/cpu/_reg_splineBasis.cpp:497-550) for a field of positions: the
// value at the clamped index, shifted by the voxel -> mm columns times the clamped distance
__device__ __forceinline__ void slided(const float *__restrict__ px, const float *__restrict__ py,
                                       const float *__restrict__ pz, int x, int y, int z, int nx, int ny, int nz,
                                       const Mat34& xyz, float& vx, float& vy, float& vz) {
    const int cx = x < 0 ? 0 : (x >= nx ? nx - 1 : x);
    const int cy = y < 0 ? 0 : (y >= ny ? ny - 1 : y);
    const int cz = z < 0 ? 0 : (z >= nz ? nz - 1 : z);
    const float sx = (float)(x - cx), sy = (float)(y - cy), sz = (float)(z - cz);
    const long long i = ((long long)cz * ny + cy) * nx + cx;
    vx = px[i] + (sx * xyz.m[0] + sy * xyz.m[1] + sz * xyz.m[2]);
    vy = py[i] + (sx * xyz.m[4] + sy * xyz.m[5] + sz * xyz.m[6]);
    vz = pz[i] + (sx * xyz.m[8] + sy * xyz.m[9] + sz * xyz.m[10]);
}

// order-preserving float <-> unsigned for atomic min / max
__device__ __forceinline__ unsigned fkey(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
float fkey_inv(unsigned k) {
    const unsigned u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

// reg_spline_getFlowFieldFromVelocityGrid (reg-lib/cpu/_reg_localTrans.cpp:3465-3491) followed by
// the displacement conversion of reg_defField_getDeformationFieldFromFlowField (:3497-3511): the
// velocity grid evaluated (cubic B-spline, composition path :903-1079) at the identity position
// of every voxel, minus that position. The 64 taps are summed as the SSE build sums them: four
// x-lanes accumulated over (z, y), then the lanes added in order. Also the extrema of all three
// components (the squaring-number rule, :3514-3521).
// One axis of the flow's sampling when the field's voxel -> mm and the grid's mm -> voxel
// matrices are both diagonal: then the identity coordinate, the grid coordinate and so the node
// index and the four basis values along an axis depend on that axis's voxel index alone (every
// off-diagonal product is an exact zero and adds nothing), and are the same floats as the
// per-voxel evaluation gives.
struct AxisEntry {
    float w[4];
    float r;  // identity coordinate (mm)
    int pre;  // first node
};

__global__ void k_axis_table(int axis, int n, FieldGeom f, Mat34 gijk, AxisEntry *__restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float fx = axis == 0 ? (float)t : 0.f, fy = axis == 1 ? (float)t : 0.f, fz = axis == 2 ? (float)t : 0.f;
    const float rx = row(f.xyz.m, fx, fy, fz), ry = row(f.xyz.m + 4, fx, fy, fz), rz = row(f.xyz.m + 8, fx, fy, fz);
    const float v = row(gijk.m + 4 * axis, rx, ry, rz);
    const int p = floor_int(v);
    const float b = v - (float)p;
    AxisEntry e;
    bspline_basis_f64(b < 0 ? 0.f : b, e.w);
    e.r = axis == 0 ? rx : (axis == 1 ? ry : rz);
    e.pre = p - 1;
    out[t] = e;
}

// at most 85 registers: three blocks of 256 threads per SM hide the tap loads' latency
template <bool kTable>
__global__ void __launch_bounds__(256, 3) k_velocity_flow(const float *__restrict__ vel, int gx, int gy, int gz,
                                                      Mat34 gxyz, Mat34 gijk, FieldGeom f,
                                                      const AxisEntry *__restrict__ tab, float *__restrict__ disp,
                                                      unsigned *__restrict__ minmax) {
    const long long n = (long long)f.nx * f.ny * f.nz;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float lo = INFINITY, hi = -INFINITY;
    if (i < n) {
        const int x = (int)(i % f.nx), y = (int)((i / f.nx) % f.ny), z = (int)(i / ((long long)f.nx * f.ny));
        float rx, ry, rz, xb[4], yb[4], zb[4];
        int xp, yp, zp;
        if (kTable) {
            const AxisEntry ex = tab[x], ey = tab[f.nx + y], ez = tab[f.nx + f.ny + z];
            rx = ex.r;
            ry = ey.r;
            rz = ez.r;
            xp = ex.pre;
            yp = ey.pre;
            zp = ez.pre;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                xb[k] = ex.w[k];
                yb[k] = ey.w[k];
                zb[k] = ez.w[k];
            }
        } else {
            const float fx = (float)x, fy = (float)y, fz = (float)z;
            rx = row(f.xyz.m, fx, fy, fz);
            ry = row(f.xyz.m + 4, fx, fy, fz);
            rz = row(f.xyz.m + 8, fx, fy, fz);
            const float vx = row(gijk.m, rx, ry, rz), vy = row(gijk.m + 4, rx, ry, rz), vz = row(gijk.m + 8, rx, ry, rz);
            xp = floor_int(vx);
            yp = floor_int(vy);
            zp = floor_int(vz);
            float b = vx - (float)xp;
            bspline_basis_f64(b < 0 ? 0.f : b, xb);
            b = vy - (float)yp;
            bspline_basis_f64(b < 0 ? 0.f : b, yb);
            b = vz - (float)zp;
            bspline_basis_f64(b < 0 ? 0.f : b, zb);
            --xp;
            --yp;
            --zp;
        }
        const long long gn = (long long)gx * gy * gz;
        const float *cx = vel, *cy = vel + gn, *cz = vel + 2 * gn;
        float tx[4] = { 0.f, 0.f, 0.f, 0.f }, ty[4] = { 0.f, 0.f, 0.f, 0.f }, tz[4] = { 0.f, 0.f, 0.f, 0.f };
        if (xp >= 0 && xp + 3 < gx && yp >= 0 && yp + 3 < gy && zp >= 0 && zp + 3 < gz) {
            // every tap inside the grid: one row pointer per (z, y), the taps in the same order
            const float *p0 = cx + ((long long)zp * gy + yp) * gx + xp;
#pragma unroll 1
            for (int c = 0; c < 4; ++c) {
#pragma unroll 1
                for (int bb = 0; bb < 4; ++bb) {
                    const float *q = p0 + (c * gy + bb) * gx;
                    const float yz = yb[bb] * zb[c];
#pragma unroll
                    for (int a = 0; a < 4; ++a) {
                        const float w = yz * xb[a];
                        tx[a] = w * __ldg(q + a) + tx[a];
                        ty[a] = w * __ldg(q + gn + a) + ty[a];
                        tz[a] = w * __ldg(q + 2 * gn + a) + tz[a];
                    }
                }
            }
        } else {
            // a border voxel: sliding values, the taps in the same order
#pragma unroll 1
            for (int c = 0; c < 4; ++c) {
#pragma unroll 1
                for (int bb = 0; bb < 4; ++bb) {
                    const float yz = yb[bb] * zb[c];
#pragma unroll
                    for (int a = 0; a < 4; ++a) {
                        const float w = yz * xb[a];
                        float px, py, pz;
                        slided(cx, cy, cz, xp + a, yp + bb, zp + c, gx, gy, gz, gxyz, px, py, pz);
                        tx[a] = w * px + tx[a];
                        ty[a] = w * py + ty[a];
                        tz[a] = w * pz + tz[a];
                    }
                }
            }
        }
        const float ox = tx[0] + tx[1] + tx[2] + tx[3];
        const float oy = ty[0] + ty[1] + ty[2] + ty[3];
        const float oz = tz[0] + tz[1] + tz[2] + tz[3];
        const float dx = ox - rx, dy = oy - ry, dz = oz - rz;
        disp[i] = dx;
        disp[n + i] = dy;
        disp[2 * n + i] = dz;
        lo = fminf(fminf(dx, dy), dz);
        hi = fmaxf(fmaxf(dx, dy), dz);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0 && lo <= hi) {
        atomicMin(minmax, fkey(lo));
        atomicMax(minmax + 1, fkey(hi));
    }
}

__global__ void k_minmax_init(unsigned *minmax) {
    minmax[0] = 0xffffffffu;
    minmax[1] = 0u;
}

// displacement / 2^N back to a deformation (reg_defField_getDeformationFieldFromFlowField,
// :3537-3547): scale is 2^-N, exact, as the reference's double division by 2^N is
__global__ void __launch_bounds__(256) k_flow_scale(float *__restrict__ d, float scale, FieldGeom f) {
    const long long n = (long long)f.nx * f.ny * f.nz;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int x = (int)(i % f.nx), y = (int)((i / f.nx) % f.ny), z = (int)(i / ((long long)f.nx * f.ny));
    const float fx = (float)x, fy = (float)y, fz = (float)z;
    d[i] = d[i] * scale + row(f.xyz.m, fx, fy, fz);
    d[n + i] = d[n + i] * scale + row(f.xyz.m + 4, fx, fy, fz);
    d[2 * n + i] = d[2 * n + i] * scale + row(f.xyz.m + 8, fx, fy, fz);
}

// reg_defField_compose3D (reg-lib/cpu/_reg_localTrans.cpp:2334-2458): out(x) = apply(pos(x)),
// trilinear in the apply field's voxel space, sliding (linear extrapolation of the positions)
// outside it. out may alias pos (each voxel reads only its own position), never apply.
constexpr int kComposeVox = 4;  // voxels per thread: their position loads and gathers overlap

__global__ void __launch_bounds__(256, 3) k_compose(const float *__restrict__ apply, const float *pos, float *out,
                                                FieldGeom f) {
    const long long n = (long long)f.nx * f.ny * f.nz;
    const long long base = (long long)blockIdx.x * blockDim.x * kComposeVox + threadIdx.x;
    const float *ax = apply, *ay = apply + n, *az = apply + 2 * n;
    float px[kComposeVox], py[kComposeVox], pz[kComposeVox];
#pragma unroll
    for (int v = 0; v < kComposeVox; ++v) {
        const long long i = base + (long long)v * blockDim.x;
        if (i < n) {
            px[v] = pos[i];
            py[v] = pos[n + i];
            pz[v] = pos[2 * n + i];
        }
    }
#pragma unroll
    for (int v = 0; v < kComposeVox; ++v) {
        const long long i = base + (long long)v * blockDim.x;
        if (i >= n) continue;
        const float vx = row(f.ijk.m, px[v], py[v], pz[v]), vy = row(f.ijk.m + 4, px[v], py[v], pz[v]),
                    vz = row(f.ijk.m + 8, px[v], py[v], pz[v]);
        const int x0 = floor_int(vx), y0 = floor_int(vy), z0 = floor_int(vz);
        float rx[2], ry[2], rz[2];
        rx[1] = vx - (float)x0;
        rx[0] = 1.f - rx[1];
        ry[1] = vy - (float)y0;
        ry[0] = 1.f - ry[1];
        rz[1] = vz - (float)z0;
        rz[0] = 1.f - rz[1];
        float ox = 0.f, oy = 0.f, oz = 0.f;
        if (x0 >= 0 && x0 + 1 < f.nx && y0 >= 0 && y0 + 1 < f.ny && z0 >= 0 && z0 + 1 < f.nz) {
            // every tap inside the field: offsets from one base, the taps in the same order
            const long long j0 = ((long long)z0 * f.ny + y0) * f.nx + x0;
            const long long sy = f.nx, sz = (long long)f.nx * f.ny;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    const long long j = j0 + c * sz + b * sy;
                    const float tb = ry[b] * rz[c];
#pragma unroll
                    for (int a = 0; a < 2; ++a) {
                        const float w = rx[a] * tb;
                        ox = ox + __ldg(ax + j + a) * w;
                        oy = oy + __ldg(ay + j + a) * w;
                        oz = oz + __ldg(az + j + a) * w;
                    }
                }
            }
        } else {
            for (int c = 0; c < 2; ++c) {
                const int z = z0 + c;
                const bool inz = z > -1 && z < f.nz;
                for (int b = 0; b < 2; ++b) {
                    const int y = y0 + b;
                    const float tb = ry[b] * rz[c];
                    const bool iny = y > -1 && y < f.ny;
                    for (int a = 0; a < 2; ++a) {
                        const int x = x0 + a;
                        float dx, dy, dz;
                        if (x > -1 && x < f.nx && iny && inz) {
                            const long long j = ((long long)z * f.ny + y) * f.nx + x;
                            dx = __ldg(ax + j);
                            dy = __ldg(ay + j);
                            dz = __ldg(az + j);
                        } else {
                            slided(ax, ay, az, x, y, z, f.nx, f.ny, f.nz, f.xyz, dx, dy, dz);
                        }
                        const float w = rx[a] * tb;
                        ox = ox + dx * w;
                        oy = oy + dy * w;
                        oz = oz + dz * w;
                    }
                }
            }
        }
        out[i] = ox;
        out[n + i] = oy;
        out[2 * n + i] = oz;
    }
}

struct Mat33f {
    float m[9];
};

// One step of Compute::ExponentiateGradient (reg-lib/Compute.cpp:288-330):
//   out = (J * trilinear(g, def(x)) + g(x)) * scale
// reg_trilinearResampleGradient (reg-lib/cpu/_reg_resampling.cpp:1537-1766) with padding 0: the
// vector image g (on the field's own grid) sampled at def(x), reoriented by the finite-difference
// Jacobian of def (forward differences, backward at the last index, where the other axes'
// differences are taken one slice back as the reference's weights select), premultiplied by
// `reorient` and divided by the real spacing per column; then reg_tools_addImageToImage, and on
// the last step the division by 2^N (scale = 2^-N, exact).
__global__ void __launch_bounds__(256) k_gradient_exp_step(const float *__restrict__ g, const float *__restrict__ def,
                                                          float *__restrict__ out, FieldGeom f, Mat33f R, float spx,
                                                          float spy, float spz, float scale) {
    const long long n = (long long)f.nx * f.ny * f.nz;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int x = (int)(i % f.nx), y = (int)((i / f.nx) % f.ny), z = (int)(i / ((long long)f.nx * f.ny));
    const float *dx = def, *dy = def + n, *dz = def + 2 * n;
    const float *gx = g, *gy = g + n, *gz = g + 2 * n;
    // sampling position in the gradient image's voxels
    const float px = dx[i], py = dy[i], pz = dz[i];
    const float cx = row(f.ijk.m, px, py, pz), cy = row(f.ijk.m + 4, px, py, pz), cz = row(f.ijk.m + 8, px, py, pz);
    int ax[2], ay[2], az[2];
    ax[0] = floor_int(cx);
    ax[1] = ceil_int(cx);
    ay[0] = floor_int(cy);
    ay[1] = ceil_int(cy);
    az[0] = floor_int(cz);
    az[1] = ceil_int(cz);
    float bx[2], by[2], bz[2];
    bx[1] = fabsf(cx - (float)ax[0]);
    by[1] = fabsf(cy - (float)ay[0]);
    bz[1] = fabsf(cz - (float)az[0]);
    bx[0] = 1.f - bx[1];
    by[0] = 1.f - by[1];
    bz[0] = 1.f - bz[1];
    float vx = 0.f, vy = 0.f, vz = 0.f;
    for (int c = 0; c < 2; ++c) {
        if (az[c] > -1 && az[c] < f.nz) {
            for (int b = 0; b < 2; ++b) {
                if (ay[b] > -1 && ay[b] < f.ny) {
                    for (int a = 0; a < 2; ++a) {
                        const float w = bx[a] * by[b] * bz[c];
                        if (ax[a] > -1 && ax[a] < f.nx) {
                            const long long j = ((long long)az[c] * f.ny + ay[b]) * f.nx + ax[a];
                            vx = vx + __ldg(gx + j) * w;
                            vy = vy + __ldg(gy + j) * w;
                            vz = vz + __ldg(gz + j) * w;
                        }
                        // a tap outside adds padding (0) * weight: nothing
                    }
                }
            }
        }
    }
    // Jacobian of the deformation by finite differences
    const int bxi = x == f.nx - 1 ? x - 1 : x, byi = y == f.ny - 1 ? y - 1 : y, bzi = z == f.nz - 1 ? z - 1 : z;
    const long long base = ((long long)bzi * f.ny + byi) * f.nx + bxi;
    const long long sx = 1, sy = f.nx, sz = (long long)f.nx * f.ny;
    float J[9];
    J[0] = dx[base + sx] - dx[base];
    J[1] = dx[base + sy] - dx[base];
    J[2] = dx[base + sz] - dx[base];
    J[3] = dy[base + sx] - dy[base];
    J[4] = dy[base + sy] - dy[base];
    J[5] = dy[base + sz] - dy[base];
    J[6] = dz[base + sx] - dz[base];
    J[7] = dz[base + sy] - dz[base];
    J[8] = dz[base + sz] - dz[base];
    // nifti_mat33_mul(reorient, J), then the division by the real spacing per column
    float M[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col)
            M[3 * r + col] = R.m[3 * r] * J[col] + R.m[3 * r + 1] * J[3 + col] + R.m[3 * r + 2] * J[6 + col];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        M[3 * r] = M[3 * r] / spx;
        M[3 * r + 1] = M[3 * r + 1] / spy;
        M[3 * r + 2] = M[3 * r + 2] / spz;
    }
    const float tx = M[0] * vx + M[1] * vy + M[2] * vz;
    const float ty = M[3] * vx + M[4] * vy + M[5] * vz;
    const float tz = M[6] * vx + M[7] * vy + M[8] * vz;
    out[i] = (tx + gx[i]) * scale;
    out[n + i] = (ty + gy[i]) * scale;
    out[2 * n + i] = (tz + gz[i]) * scale;
}

// Compute::SymmetriseVelocityFields (reg-lib/Compute.cpp:356-392): both grids as displacements,
// forward = (fw - bw) / 2, backward = (bw - fw) / 2, back to positions. Both grids share dims.
__global__ void __launch_bounds__(256) k_symmetrise(float *__restrict__ fw, float *__restrict__ bw, int nx, int ny,
                                                   int nz, Mat34 fxyz, Mat34 bxyz) {
    const long long n = (long long)nx * ny * nz;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long long)nx * ny));
    const float fx = (float)x, fy = (float)y, fz = (float)z;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float idf = row(fxyz.m + 4 * k, fx, fy, fz), idb = row(bxyz.m + 4 * k, fx, fy, fz);
        const float df = fw[k * n + i] - idf, db = bw[k * n + i] - idb;
        fw[k * n + i] = (df - db) * 0.5f + idf;
        bw[k * n + i] = (db - df) * 0.5f + idb;
    }
}

// reg_voxelCentricToNodeCentric (reg-lib/cpu/_reg_localTrans.cpp:1540-1685) for a grid in any
// orientation relative to the image: each node mapped into the image's voxels (T = image ijk x
// grid xyz, Mat44Mul in double), the convolved voxel gradient sampled trilinearly (0 outside),
// reoriented by the transpose of R and scaled by the weight. One thread per node.
__global__ void k_voxel_to_node_general(const float *__restrict__ vox, int nx, int ny, int nz, Mat34 T, Mat33f R,
                                        float weight, int cx, int cy, int cz, float *__restrict__ node) {
    const long long nc = (long long)cx * cy * cz, nv = (long long)nx * ny * nz;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nc) return;
    const double gx = (double)(i % cx), gy = (double)((i / cx) % cy), gz = (double)(i / ((long long)cx * cy));
    float v[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
        v[r] = (float)((double)T.m[4 * r] * gx + (double)T.m[4 * r + 1] * gy + (double)T.m[4 * r + 2] * gz +
                       (double)T.m[4 * r + 3]);
    int pre[3];
    float b[3][2];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        pre[k] = floor_int(v[k]);
        b[k][1] = v[k] - (float)pre[k];
        b[k][0] = 1.f - b[k][1];
    }
    float iv0 = 0.f, iv1 = 0.f, iv2 = 0.f;
    for (int c = 0; c < 2; ++c) {
        const int Z = pre[2] + c;
        if (Z <= -1 || Z >= nz) continue;
        for (int bb = 0; bb < 2; ++bb) {
            const int Y = pre[1] + bb;
            if (Y <= -1 || Y >= ny) continue;
            for (int a = 0; a < 2; ++a) {
                const int X = pre[0] + a;
                if (X <= -1 || X >= nx) continue;
                const long long j = ((long long)Z * ny + Y) * nx + X;
                float lw = b[0][a] * b[1][bb];
                lw = lw * b[2][c];
                iv0 = iv0 + lw * __ldg(vox + j);
                iv1 = iv1 + lw * __ldg(vox + nv + j);
                iv2 = iv2 + lw * __ldg(vox + 2 * nv + j);
            }
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float ro = R.m[d] * iv0 + R.m[3 + d] * iv1 + R.m[6 + d] * iv2;
        node[d * nc + i] = ro * weight;
    }
}

inline unsigned blocks_for(long long n) { return (unsigned)((n + 255) / 256); }
inline unsigned compose_blocks(long long n) { return (unsigned)((n + 256LL * kComposeVox - 1) / (256LL * kComposeVox)); }

// algorithmic bytes of one composition per voxel: its position read, the applied field read once
// and the result written, 3 x 4 bytes each; a squaring step applies the field to itself, so the
// positions and the applied field are one read
constexpr double kComposeBytes = 36.0, kSquaringBytes = 24.0;

}  // namespace

// The squaring-number rule of reg_defField_getDeformationFieldFromFlowField (:3514-3526): the
// smallest N with max|displacement| / 2^N < 0.28 (3D), at least 6.
int velocity_squaring_steps(float vmin, float vmax) {
    float extrema = std::max(std::fabs(vmin), vmax);
    int steps = 1;
    while (extrema / static_cast<float>(std::pow(2, steps)) >= 0.28f) ++steps;
    return std::max(steps, 6);
}

// reg_spline_getDefFieldFromVelocityGrid (reg-lib/cpu/_reg_localTrans.cpp:3583-3613) and
// reg_spline_getIntermediateDefFieldFromVelGrid (:3616-3681) on the field grid g->ref_* from the
// velocity grid g->cpp_*. *steps is the grid's squaring number (its intent_p2); with update it is
// first recomputed from this flow (a host read of the extrema). def (optional) receives the
// exponentiated field; fields (optional) the fields after 0..N-1 squarings, N * 3 * nvox floats.
// scratch: 3 * nvox floats; minmax: 2 unsigned on the device.
nrb_status velocity_to_deformation(const nrb_geometry *g, const float *vel, bool update, int *steps, float *def,
                                   float *fields, float *scratch, unsigned *minmax, cudaStream_t st) {
    const FieldGeom f = field_geom(g->ref_dim, g->ref_xyz, g->ref_ijk);
    const long long n = nvox(g->ref_dim);
    if (!def && !fields) return fail(NRB_ERR_INVALID, "velocity exponentiation: no output");
    KernelTimer stage(TK_F2_VELOCITY, 0.0, st);
    int N = *steps;
    // the flow (displacement) lands where the squarings start: the first intermediate field, or
    // the buffer from which N ping-pong squarings end in def
    float *first = fields ? fields : (N % 2 == 0 ? def : scratch);
    if (update) {
        k_minmax_init<<<1, 1, 0, st>>>(minmax);
        NRB_LAUNCHED("k_minmax_init");
    }
    auto diagonal = [](const float *m) {
        return m[1] == 0.f && m[2] == 0.f && m[4] == 0.f && m[6] == 0.f && m[8] == 0.f && m[9] == 0.f;
    };
    if (diagonal(g->ref_xyz) && diagonal(g->cpp_ijk)) {
        const int nt = f.nx + f.ny + f.nz;
        AxisEntry *tab = nullptr;
        NRB_CUDA(dev_alloc(&tab, nt * sizeof(AxisEntry), st));
        const int off[3] = { 0, f.nx, f.nx + f.ny }, len[3] = { f.nx, f.ny, f.nz };
        for (int a = 0; a < 3; ++a) {
            k_axis_table<<<(len[a] + 127) / 128, 128, 0, st>>>(a, len[a], f, to_mat34(g->cpp_ijk), tab + off[a]);
            NRB_LAUNCHED("k_axis_table");
        }
        k_velocity_flow<true><<<blocks_for(n), 256, 0, st>>>(vel, g->cpp_dim[0], g->cpp_dim[1], g->cpp_dim[2],
                                                             to_mat34(g->cpp_xyz), to_mat34(g->cpp_ijk), f, tab,
                                                             first, minmax);
        dev_free(tab, st);
    } else {
        k_velocity_flow<false><<<blocks_for(n), 256, 0, st>>>(vel, g->cpp_dim[0], g->cpp_dim[1], g->cpp_dim[2],
                                                              to_mat34(g->cpp_xyz), to_mat34(g->cpp_ijk), f, nullptr,
                                                              first, minmax);
    }
    NRB_LAUNCHED("k_velocity_flow");
    if (update) {
        // the extrema land in pinned host memory (a pageable copy would stage through the driver):
        // 8 bytes per host thread, portable across devices, kept for the thread's lifetime
        static thread_local unsigned *mm = nullptr;
        if (!mm) NRB_CUDA(cudaHostAlloc((void **)&mm, 2 * sizeof(unsigned), cudaHostAllocPortable));
        NRB_CUDA(cudaMemcpyAsync(mm, minmax, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        NRB_CUDA(cudaStreamSynchronize(st));
        N = velocity_squaring_steps(fkey_inv(mm[0]), fkey_inv(mm[1]));
        *steps = N;
        if (def && !fields && first != (N % 2 == 0 ? def : scratch)) {
            // the parity of N changed: move the flow to where an even or odd chain ends in def
            float *want = N % 2 == 0 ? def : scratch;
            NRB_CUDA(cudaMemcpyAsync(want, first, 3 * n * sizeof(float), cudaMemcpyDeviceToDevice, st));
            first = want;
        }
    }
    k_flow_scale<<<blocks_for(n), 256, 0, st>>>(first, std::ldexp(1.f, -N), f);
    NRB_LAUNCHED("k_flow_scale");
    if (fields) {
        // keep every intermediate field; the last squaring only when def is wanted
        for (int k = 1; k < N; ++k) {
            KernelTimer kt(TK_F2_COMPOSE, kSquaringBytes * n, st);
            k_compose<<<compose_blocks(n), 256, 0, st>>>(fields + (k - 1) * 3 * n, fields + (k - 1) * 3 * n,
                                                     fields + k * 3 * n, f);
            NRB_LAUNCHED("k_compose");
        }
        if (def) {
            KernelTimer kt(TK_F2_COMPOSE, kSquaringBytes * n, st);
            k_compose<<<compose_blocks(n), 256, 0, st>>>(fields + (N - 1) * 3 * n, fields + (N - 1) * 3 * n, def, f);
            NRB_LAUNCHED("k_compose");
        }
        return NRB_OK;
    }
    float *a = first, *b = first == def ? scratch : def;
    for (int k = 0; k < N; ++k) {
        KernelTimer kt(TK_F2_COMPOSE, kSquaringBytes * n, st);
        k_compose<<<compose_blocks(n), 256, 0, st>>>(a, a, b, f);
        NRB_LAUNCHED("k_compose");
        std::swap(a, b);
    }
    return NRB_OK;  // a == def after N swaps
}

nrb_status compose_fields(const int32_t dim[3], const float xyz[16], const float ijk[16], const float *apply,
                          float *update, cudaStream_t st) {
    const FieldGeom f = field_geom(dim, xyz, ijk);
    KernelTimer kt(TK_F2_COMPOSE, kComposeBytes * nvox(dim), st);
    k_compose<<<compose_blocks(nvox(dim)), 256, 0, st>>>(apply, update, update, f);
    NRB_LAUNCHED("k_compose");
    return NRB_OK;
}

// nifti_mat33_polar's role (the orthogonal factor of a 3x3 matrix) by Higham's scaled Newton
// iteration, in double
static void polar_factor(const double A[3][3], double Q[3][3]) {
    double X[3][3];
    memcpy(X, A, sizeof(X));
    for (int it = 0; it < 100; ++it) {
        const double det = X[0][0] * (X[1][1] * X[2][2] - X[1][2] * X[2][1]) -
                           X[0][1] * (X[1][0] * X[2][2] - X[1][2] * X[2][0]) +
                           X[0][2] * (X[1][0] * X[2][1] - X[1][1] * X[2][0]);
        if (det == 0.0) break;
        double Y[3][3];  // inverse transpose
        Y[0][0] = (X[1][1] * X[2][2] - X[1][2] * X[2][1]) / det;
        Y[0][1] = (X[1][2] * X[2][0] - X[1][0] * X[2][2]) / det;
        Y[0][2] = (X[1][0] * X[2][1] - X[1][1] * X[2][0]) / det;
        Y[1][0] = (X[0][2] * X[2][1] - X[0][1] * X[2][2]) / det;
        Y[1][1] = (X[0][0] * X[2][2] - X[0][2] * X[2][0]) / det;
        Y[1][2] = (X[0][1] * X[2][0] - X[0][0] * X[2][1]) / det;
        Y[2][0] = (X[0][1] * X[1][2] - X[0][2] * X[1][1]) / det;
        Y[2][1] = (X[0][2] * X[1][0] - X[0][0] * X[1][2]) / det;
        Y[2][2] = (X[0][0] * X[1][1] - X[0][1] * X[1][0]) / det;
        double nx = 0, ny = 0;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                nx += X[r][c] * X[r][c];
                ny += Y[r][c] * Y[r][c];
            }
        const double gam = std::sqrt(std::sqrt(ny / nx));
        double d = 0;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                const double v = 0.5 * (gam * X[r][c] + Y[r][c] / gam);
                d += std::fabs(v - X[r][c]);
                X[r][c] = v;
            }
        if (d < 1e-15) break;
    }
    memcpy(Q, X, sizeof(X));
}

// reg_getRealImageSpacing (reg-lib/cpu/_reg_tools.cpp:253-273): the distance in mm between voxel
// 0 and its neighbour along each axis, through Mat44Mul (double, rounded to float)
static void real_spacing(const float xyz[16], float sp[3]) {
    float o[3];
    for (int r = 0; r < 3; ++r) o[r] = (float)((double)xyz[4 * r + 3]);
    for (int c = 0; c < 3; ++c) {
        float p[3];
        for (int r = 0; r < 3; ++r) p[r] = (float)((double)xyz[4 * r + c] + (double)xyz[4 * r + 3]);
        const float a = o[0] - p[0], b = o[1] - p[1], d = o[2] - p[2];
        sp[c] = std::sqrt(a * a + b * b + d * d);
    }
}

// Compute::ExponentiateGradient (reg-lib/Compute.cpp:288-330) for the voxel-based gradient
// `vgrad` on g->ref_* and the opposite transformation's velocity grid g->cpp_*: the intermediate
// fields of that grid (N squarings), then N gradient resampling steps, then the division by 2^N.
// fields: N * 3 * nvox floats, scratch: 3 * nvox floats.
nrb_status exponentiate_gradient(const nrb_geometry *g, const float *vel_other, int steps, float *vgrad,
                                 float *fields, float *scratch, unsigned *minmax, cudaStream_t st) {
    if (steps < 1) return fail(NRB_ERR_INVALID, "gradient exponentiation: the squaring number must be >= 1");
    KernelTimer stage(TK_F2_GRADIENT_EXP, 0.0, st);
    int N = steps;
    NRB_TRY(velocity_to_deformation(g, vel_other, false, &N, nullptr, fields, scratch, minmax, st));
    const FieldGeom f = field_geom(g->ref_dim, g->ref_xyz, g->ref_ijk);
    const long long n = nvox(g->ref_dim);
    // reorient = inverse(polar(rotation-scaling part of voxel -> mm))
    double A[3][3], Q[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) A[r][c] = g->ref_xyz[4 * r + c];
    polar_factor(A, Q);
    Mat33f R;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) R.m[3 * r + c] = (float)Q[c][r];  // inverse of an orthogonal matrix
    float sp[3];
    real_spacing(g->ref_xyz, sp);
    float *a = vgrad, *b = scratch;
    for (int k = 0; k < N; ++k) {
        const float scale = k == N - 1 ? std::ldexp(1.f, -N) : 1.f;
        k_gradient_exp_step<<<blocks_for(n), 256, 0, st>>>(a, fields + (long long)k * 3 * n, b, f, R, sp[0], sp[1],
                                                           sp[2], scale);
        NRB_LAUNCHED("k_gradient_exp_step");
        std::swap(a, b);
    }
    if (a != vgrad) NRB_CUDA(cudaMemcpyAsync(vgrad, a, 3 * n * sizeof(float), cudaMemcpyDeviceToDevice, st));
    return NRB_OK;
}

// The voxel -> node step for a grid not aligned with the image (the F3D2 grids of rotated
// images): `vox` holds the voxel gradient already convolved along the image axes.
nrb_status voxel_to_node_general(const float *vox, const nrb_geometry *g, float weight, float *node,
                                 cudaStream_t st) {
    float T[16];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            double acc = 0;
            for (int k = 0; k < 4; ++k) acc += (double)g->ref_ijk[4 * r + k] * (double)g->cpp_xyz[4 * k + c];
            T[4 * r + c] = (float)acc;  // mat44 product, each entry rounded to float
        }
    for (int r = 0; r < 3; ++r) {
        const float a = g->cpp_xyz[4 * r], b = g->cpp_xyz[4 * r + 1], c = g->cpp_xyz[4 * r + 2];
        float ratio = std::sqrt(a * a + b * b + c * c);
        ratio = ratio / g->ref_pixdim[r];
        weight = weight * ratio;
    }
    Mat33f R;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) R.m[3 * r + c] = g->flo_ijk[4 * r + c];
    const long long nc = nvox(g->cpp_dim);
    k_voxel_to_node_general<<<blocks_for(nc), 256, 0, st>>>(vox, g->ref_dim[0], g->ref_dim[1], g->ref_dim[2],
                                                           to_mat34(T), R, weight, g->cpp_dim[0], g->cpp_dim[1],
                                                           g->cpp_dim[2], node);
    NRB_LAUNCHED("k_voxel_to_node_general");
    return NRB_OK;
}

nrb_status symmetrise_velocity(const int32_t cdim[3], const float fw_xyz[16], float *fw, const float bw_xyz[16],
                               float *bw, cudaStream_t st) {
    k_symmetrise<<<blocks_for(nvox(cdim)), 256, 0, st>>>(fw, bw, cdim[0], cdim[1], cdim[2], to_mat34(fw_xyz),
                                                         to_mat34(bw_xyz));
    NRB_LAUNCHED("k_symmetrise");
    return NRB_OK;
}

}  // namespace nrb

using namespace nrb;

static nrb_status check_field_geometry(const nrb_geometry *g, const char *what) {
    for (int i = 0; i < 3; ++i)
        if (g->ref_dim[i] < 1 || g->cpp_dim[i] < 1) return fail(NRB_ERR_INVALID, std::string(what) + ": empty grid");
    if (nvox(g->ref_dim) >= (1LL << 40) || nvox(g->cpp_dim) >= (1LL << 40))
        return fail(NRB_ERR_UNSUPPORTED, std::string(what) + ": grid too large");
    return NRB_OK;
}

// scratch buffers of one call, freed in stream order
struct Scratch {
    float *p = nullptr;
    unsigned *mm = nullptr;
    cudaStream_t st;
    explicit Scratch(cudaStream_t s): st(s) {}
    ~Scratch() {
        dev_free(p, st);
        dev_free(mm, st);
    }
};

extern "C" nrb_status nrb_get_def_field_from_velocity_grid(const nrb_geometry *g, const float *vel,
                                                          int update_step_number, int32_t *steps, float *def,
                                                          void *stream) {
    if (!g || !vel || !steps || !def) return fail(NRB_ERR_INVALID, "nrb_get_def_field_from_velocity_grid: null pointer");
    NRB_TRY(check_field_geometry(g, "nrb_get_def_field_from_velocity_grid"));
    if (*steps < 1 && !update_step_number)
        return fail(NRB_ERR_INVALID, "nrb_get_def_field_from_velocity_grid: the squaring number must be >= 1");
    cudaStream_t st = as_stream(stream);
    Scratch s(st);
    NRB_CUDA(dev_alloc(&s.p, 3 * nvox(g->ref_dim) * sizeof(float), st));
    NRB_CUDA(dev_alloc(&s.mm, 2 * sizeof(unsigned), st));
    int N = *steps < 1 ? 6 : *steps;
    NRB_TRY(velocity_to_deformation(g, vel, update_step_number != 0 || *steps == 0, &N, def, nullptr, s.p, s.mm, st));
    *steps = N;
    return NRB_OK;
}

extern "C" nrb_status nrb_def_field_compose(const int32_t dim[3], const float xyz[16], const float ijk[16],
                                           const float *apply, float *update, void *stream) {
    if (!dim || !xyz || !ijk || !apply || !update) return fail(NRB_ERR_INVALID, "nrb_def_field_compose: null pointer");
    if (apply == update) return fail(NRB_ERR_INVALID, "nrb_def_field_compose: the two fields must not alias");
    for (int i = 0; i < 3; ++i)
        if (dim[i] < 1) return fail(NRB_ERR_INVALID, "nrb_def_field_compose: empty field");
    return compose_fields(dim, xyz, ijk, apply, update, as_stream(stream));
}

extern "C" nrb_status nrb_exponentiate_gradient(const nrb_geometry *g, const float *vel_other, int32_t steps,
                                               float *vgrad, void *stream) {
    if (!g || !vel_other || !vgrad) return fail(NRB_ERR_INVALID, "nrb_exponentiate_gradient: null pointer");
    NRB_TRY(check_field_geometry(g, "nrb_exponentiate_gradient"));
    for (int i = 0; i < 3; ++i)  // the Jacobian's finite differences need two voxels per axis
        if (g->ref_dim[i] < 2) return fail(NRB_ERR_INVALID, "nrb_exponentiate_gradient: 3D fields of >= 2 voxels per axis");
    if (steps < 1 || steps > 30) return fail(NRB_ERR_INVALID, "nrb_exponentiate_gradient: squaring number in [1, 30]");
    cudaStream_t st = as_stream(stream);
    const long long n = nvox(g->ref_dim);
    Scratch s(st), fields(st);
    NRB_CUDA(dev_alloc(&s.p, 3 * n * sizeof(float), st));
    NRB_CUDA(dev_alloc(&s.mm, 2 * sizeof(unsigned), st));
    NRB_CUDA(dev_alloc(&fields.p, (size_t)steps * 3 * n * sizeof(float), st));
    return exponentiate_gradient(g, vel_other, steps, vgrad, fields.p, s.p, s.mm, st);
}

extern "C" nrb_status nrb_symmetrise_velocity_fields(const nrb_geometry *g_fw, float *fw, const nrb_geometry *g_bw,
                                                    float *bw, void *stream) {
    if (!g_fw || !fw || !g_bw || !bw) return fail(NRB_ERR_INVALID, "nrb_symmetrise_velocity_fields: null pointer");
    for (int i = 0; i < 3; ++i)
        if (g_fw->cpp_dim[i] != g_bw->cpp_dim[i] || g_fw->cpp_dim[i] < 1)
            return fail(NRB_ERR_INVALID, "nrb_symmetrise_velocity_fields: the two grids must have the same dims");
    if (fw == bw) return fail(NRB_ERR_INVALID, "nrb_symmetrise_velocity_fields: the two grids must not alias");
    return symmetrise_velocity(g_fw->cpp_dim, g_fw->cpp_xyz, fw, g_bw->cpp_xyz, bw, as_stream(stream));
}
