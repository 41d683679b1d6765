// Voxel-pass kernels of the F3D objective and gradient.
//
// Every kernel here walks the reference volume in 32x4x4-voxel tiles. For a tile, the block of
// control points its voxels depend on is staged in shared memory and the cubic B-spline sum
// sum_{a,b,c} Bx_a By_b Bz_c CP is evaluated separably (z, then y, then x), about 21 FMAs per
// voxel instead of 192. The deformation field never leaves the SM in the fused kernels: it is
// consumed at once by the trilinear warp, the joint histogram (objective) or the spatial
// gradient and NMI voxel gradient (gradient).
#include <cfloat>
#include <cmath>

#include "nrb_state.cuh"

namespace nrb {

struct TileParams {
    int nx, ny, nz;          // reference / deformation-field dims
    int cx, cy, cz;          // control-point grid dims
    float gsx, gsy, gsz;     // grid spacing in reference voxels (grid pixdim / ref pixdim)
    int sa, sb, sc;          // shared-memory strides: max node span of a tile per axis
    int tiles_x, tiles_y, tiles_z, ntiles;
    int fnx, fny, fnz;       // floating dims
    Mat34 flo_ijk;           // mm -> floating voxel
    float pad;               // padding value of out-of-volume taps
    int rb, fb;              // internal bin counts
    int tile_floats;         // shared floats used by the tile machinery
    long long cnv;           // control points per component
};

__device__ __forceinline__ int pre_of(int v, float gs) { return (int)((float)v / gs); }

__device__ __forceinline__ float frac_of(int v, float gs, int pre) {
    const float t = (float)v / gs - (float)pre;
    return t < 0.f ? 0.f : t;
}

// Shared-memory layout of one tile (in floats):
//   cp  [3][sc][sb][sa]  control points minus the tile offset; later reused for
//   r   [3][TZ][TY][sa]  the y- and z-contracted sums
//   q   [3][TZ][sb][sa]  the z-contracted sums
//   bz[TZ][4], by[TY][4], zo[TZ], yo[TY], off[3]
__host__ __device__ inline int tile_smem_floats(int sa, int sb, int sc) {
    return 3 * sc * sb * sa + 3 * TILE_Z * sb * sa + TILE_Z * 4 + TILE_Y * 4 + TILE_Z + TILE_Y + 4;
}

struct TileCtx {
    int x0, y0, z0, xa0, yb0, zc0;
};

// Stages the control points of `tile` and leaves the y/z-contracted sums r[c][z'][y'][a] and
// the offsets in shared memory. Must be called by all threads of the block.
__device__ void tile_positions(const TileParams& P, const float *__restrict__ cpp, int tile,
                               float *sm, TileCtx& T) {
    const int tid = threadIdx.x;
    const int tx = tile % P.tiles_x;
    const int t2 = tile / P.tiles_x;
    const int ty = t2 % P.tiles_y;
    const int tz = t2 / P.tiles_y;
    T.x0 = tx * TILE_X;
    T.y0 = ty * TILE_Y;
    T.z0 = tz * TILE_Z;
    T.xa0 = pre_of(T.x0, P.gsx);
    T.yb0 = pre_of(T.y0, P.gsy);
    T.zc0 = pre_of(T.z0, P.gsz);
    const int na = pre_of(min(T.x0 + TILE_X - 1, P.nx - 1), P.gsx) + 4 - T.xa0;
    const int nb = pre_of(min(T.y0 + TILE_Y - 1, P.ny - 1), P.gsy) + 4 - T.yb0;
    const int nc = pre_of(min(T.z0 + TILE_Z - 1, P.nz - 1), P.gsz) + 4 - T.zc0;

    float *cp = sm;
    float *q = sm + 3 * P.sc * P.sb * P.sa;
    float *bz = q + 3 * TILE_Z * P.sb * P.sa;
    float *by = bz + TILE_Z * 4;
    int *zo = reinterpret_cast<int *>(by + TILE_Y * 4);
    int *yo = zo + TILE_Z;
    float *off = reinterpret_cast<float *>(yo + TILE_Y);

    __syncthreads();  // the previous tile's readers are done with r / off
    const long long cnv = P.cnv;
    if (tid < 3) off[tid] = __ldg(&cpp[tid * cnv + ((long long)T.zc0 * P.cy + T.yb0) * P.cx + T.xa0]);
    if (tid >= 32 && tid < 32 + TILE_Z) {
        const int zp = tid - 32, z = T.z0 + zp;
        const int pre = pre_of(min(z, P.nz - 1), P.gsz);
        zo[zp] = pre - T.zc0;
        bspline_basis(frac_of(min(z, P.nz - 1), P.gsz, pre), bz + 4 * zp);
    }
    if (tid >= 64 && tid < 64 + TILE_Y) {
        const int yp = tid - 64, y = T.y0 + yp;
        const int pre = pre_of(min(y, P.ny - 1), P.gsy);
        yo[yp] = pre - T.yb0;
        bspline_basis(frac_of(min(y, P.ny - 1), P.gsy, pre), by + 4 * yp);
    }
    __syncthreads();
    // stage the control-point block (relative to the tile offset, which keeps the magnitudes
    // of the partial sums small)
    const int ncp = 3 * nc * nb * na;
    for (int i = tid; i < ncp; i += TILE_THREADS) {
        const int ia = i % na;
        int rest = i / na;
        const int jb = rest % nb;
        rest /= nb;
        const int kc = rest % nc;
        const int c = rest / nc;
        const float v = __ldg(&cpp[c * cnv + ((long long)(T.zc0 + kc) * P.cy + (T.yb0 + jb)) * P.cx + T.xa0 + ia]);
        cp[((c * P.sc + kc) * P.sb + jb) * P.sa + ia] = v - off[c];
    }
    __syncthreads();
    // z contraction
    const int nq = 3 * TILE_Z * nb * na;
    for (int i = tid; i < nq; i += TILE_THREADS) {
        const int ia = i % na;
        int rest = i / na;
        const int jb = rest % nb;
        rest /= nb;
        const int zp = rest % TILE_Z;
        const int c = rest / TILE_Z;
        const float *src = cp + ((c * P.sc + zo[zp]) * P.sb + jb) * P.sa + ia;
        const float *w = bz + 4 * zp;
        const int st = P.sb * P.sa;
        float s = w[0] * src[0];
        s = fmaf(w[1], src[st], s);
        s = fmaf(w[2], src[2 * st], s);
        s = fmaf(w[3], src[3 * st], s);
        q[((c * TILE_Z + zp) * P.sb + jb) * P.sa + ia] = s;
    }
    __syncthreads();
    // y contraction into r (aliases cp, which is dead now)
    float *r = cp;
    const int nr = 3 * TILE_Z * TILE_Y * na;
    for (int i = tid; i < nr; i += TILE_THREADS) {
        const int ia = i % na;
        int rest = i / na;
        const int yp = rest % TILE_Y;
        rest /= TILE_Y;
        const int zp = rest % TILE_Z;
        const int c = rest / TILE_Z;
        const float *src = q + ((c * TILE_Z + zp) * P.sb + yo[yp]) * P.sa + ia;
        const float *w = by + 4 * yp;
        float s = w[0] * src[0];
        s = fmaf(w[1], src[P.sa], s);
        s = fmaf(w[2], src[2 * P.sa], s);
        s = fmaf(w[3], src[3 * P.sa], s);
        r[((c * TILE_Z + zp) * TILE_Y + yp) * P.sa + ia] = s;
    }
    __syncthreads();
}

__device__ __forceinline__ const float *tile_offsets(const TileParams& P, const float *sm) {
    const float *q = sm + 3 * P.sc * P.sb * P.sa;
    const float *bz = q + 3 * TILE_Z * P.sb * P.sa;
    return bz + TILE_Z * 4 + TILE_Y * 4 + TILE_Z + TILE_Y;
}

// Final x contraction for voxel (lx, ly, zp) of the tile: world position in mm.
__device__ __forceinline__ void voxel_position(const TileParams& P, const float *sm,
                                               const float *off, int ly, int zp, int xo,
                                               const float bx[4], float& px, float& py,
                                               float& pz) {
    const int cs = TILE_Z * TILE_Y * P.sa;
    const float *r = sm + (zp * TILE_Y + ly) * P.sa + xo;
    float s0 = bx[0] * r[0], s1 = bx[0] * r[cs], s2 = bx[0] * r[2 * cs];
#pragma unroll
    for (int t = 1; t < 4; ++t) {
        s0 = fmaf(bx[t], r[t], s0);
        s1 = fmaf(bx[t], r[cs + t], s1);
        s2 = fmaf(bx[t], r[2 * cs + t], s2);
    }
    px = off[0] + s0;
    py = off[1] + s1;
    pz = off[2] + s2;
}

// mm -> floating voxel as Mat44Mul does it (reg-lib/cpu/Maths.hpp:272-286): the products of
// two floats are exact in double, the sum is rounded once to double and then to float.
__device__ __forceinline__ void to_floating_voxel(const Mat34& M, float x, float y, float z,
                                                  float& fx, float& fy, float& fz) {
    const double dx = x, dy = y, dz = z;
    fx = (float)((double)M.m[0] * dx + (double)M.m[1] * dy + (double)M.m[2] * dz + (double)M.m[3]);
    fy = (float)((double)M.m[4] * dx + (double)M.m[5] * dy + (double)M.m[6] * dz + (double)M.m[7]);
    fz = (float)((double)M.m[8] * dx + (double)M.m[9] * dy + (double)M.m[10] * dz + (double)M.m[11]);
}

// Trilinear sample of the floating image at world position (x, y, z) with the padding rule of
// ResampleImage3D (an out-of-volume tap contributes padding * weight) and, when kGrad, the
// spatial derivative of TrilinearImageGradient (NaN components -> 0).
template <bool kGrad>
__device__ __forceinline__ void sample_floating(const float *__restrict__ flo, int fnx, int fny,
                                                int fnz, const Mat34& M, float pad, float x,
                                                float y, float z, float& val, float g[3]) {
    float fx, fy, fz;
    to_floating_voxel(M, x, y, z, fx, fy, fz);
    const int px = (int)floorf(fx), py = (int)floorf(fy), pz = (int)floorf(fz);
    const float rx = fx - (float)px, ry = fy - (float)py, rz = fz - (float)pz;
    const float bx0 = 1.f - rx, by0 = 1.f - ry, bz0 = 1.f - rz;
    float v[2][2][2];
    const bool interior = px >= 0 && py >= 0 && pz >= 0 && px + 1 < fnx && py + 1 < fny && pz + 1 < fnz;
    if (interior) {
        const float *p = flo + ((long long)pz * fny + py) * fnx + px;
        const long long sy = fnx, sz = (long long)fnx * fny;
        v[0][0][0] = __ldg(p);
        v[0][0][1] = __ldg(p + 1);
        v[0][1][0] = __ldg(p + sy);
        v[0][1][1] = __ldg(p + sy + 1);
        v[1][0][0] = __ldg(p + sz);
        v[1][0][1] = __ldg(p + sz + 1);
        v[1][1][0] = __ldg(p + sz + sy);
        v[1][1][1] = __ldg(p + sz + sy + 1);
    } else {
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    const int X = px + a, Y = py + b, Z = pz + c;
                    const bool in = X >= 0 && X < fnx && Y >= 0 && Y < fny && Z >= 0 && Z < fnz;
                    v[c][b][a] = in ? __ldg(&flo[((long long)Z * fny + Y) * fnx + X]) : pad;
                }
    }
    float yv0 = fmaf(v[0][0][1], rx, v[0][0][0] * bx0);
    float yv1 = fmaf(v[0][1][1], rx, v[0][1][0] * bx0);
    const float zv0 = fmaf(yv1, ry, yv0 * by0);
    float yw0 = fmaf(v[1][0][1], rx, v[1][0][0] * bx0);
    float yw1 = fmaf(v[1][1][1], rx, v[1][1][0] * bx0);
    const float zv1 = fmaf(yw1, ry, yw0 * by0);
    val = fmaf(zv1, rz, zv0 * bz0);
    if (kGrad) {
        // d/dx: (v1 - v0) along x, weighted by y and z; d/dy, d/dz from the x-interpolated rows
        const float dx00 = v[0][0][1] - v[0][0][0], dx01 = v[0][1][1] - v[0][1][0];
        const float dx10 = v[1][0][1] - v[1][0][0], dx11 = v[1][1][1] - v[1][1][0];
        const float gx0 = fmaf(dx01, ry, dx00 * by0), gx1 = fmaf(dx11, ry, dx10 * by0);
        g[0] = fmaf(gx1, rz, gx0 * bz0);
        g[1] = fmaf(yw1 - yw0, rz, (yv1 - yv0) * bz0);
        g[2] = zv1 - zv0;
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (g[d] != g[d]) g[d] = 0.f;
    }
}

// ---------------------------------------------------------------------------------------------
// fused objective: deformation + warp + joint histogram
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(TILE_THREADS)
k_objective(TileParams P, const float *__restrict__ ref, const float *__restrict__ flo,
            const int32_t *__restrict__ mask, const float *__restrict__ cpp,
            uint32_t *__restrict__ ghist) {
    extern __shared__ float4 sm4[];
    float *sm = reinterpret_cast<float *>(sm4);
    uint32_t *h = reinterpret_cast<uint32_t *>(sm + P.tile_floats);
    const int nbins = P.rb * P.fb;
    for (int i = threadIdx.x; i < nbins; i += TILE_THREADS) h[i] = 0u;
    const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
    for (int tile = blockIdx.x; tile < P.ntiles; tile += gridDim.x) {
        TileCtx T;
        tile_positions(P, cpp, tile, sm, T);
        const float *off = tile_offsets(P, sm);
        const int x = T.x0 + lx, y = T.y0 + ly;
        const bool xyin = x < P.nx && y < P.ny;
        float bx[4] = { 0, 0, 0, 0 };
        int xo = 0;
        if (xyin) {
            const int pre = pre_of(x, P.gsx);
            bspline_basis(frac_of(x, P.gsx, pre), bx);
            xo = pre - T.xa0;
        }
#pragma unroll 1
        for (int zp = 0; zp < TILE_Z; ++zp) {
            const int z = T.z0 + zp;
            int bin = -1;
            if (xyin && z < P.nz) {
                const long long idx = ((long long)z * P.ny + y) * P.nx + x;
                if (mask == nullptr || __ldg(&mask[idx]) > -1) {
                    float wx, wy, wz, w, g[3];
                    voxel_position(P, sm, off, ly, zp, xo, bx, wx, wy, wz);
                    sample_floating<false>(flo, P.fnx, P.fny, P.fnz, P.flo_ijk, P.pad, wx, wy, wz, w, g);
                    const float rv = __ldg(&ref[idx]);
                    if (rv == rv && w == w && 0.f <= rv && rv < (float)P.rb && 0.f <= w && w < (float)P.fb)
                        bin = (int)rv + (int)w * P.rb;
                }
            }
            // warp-aggregated shared-memory increment: one atomic per distinct bin
            const unsigned peers = __match_any_sync(0xffffffffu, bin);
            if (bin >= 0 && lx == __ffs(peers) - 1) atomicAdd(&h[bin], (uint32_t)__popc(peers));
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nbins; i += TILE_THREADS) {
        const uint32_t v = h[i];
        if (v) atomicAdd(&ghist[i], v);
    }
}

// Sum over the 4x4 Parzen window of reg_getVoxelBasedNmiGradient3d (_reg_nmi.cpp:548-571):
// returns refDeriv + warDeriv - nmi * jointDeriv for a unit spatial gradient.
__device__ __forceinline__ double nmi_window(float rv, float wv, const double *__restrict__ logt,
                                             int rb, int fb, double nmi) {
    const double *rlog = logt + rb * fb;
    const double *wlog = rlog + rb;
    double sr = 0, sw = 0, sj = 0;
    const int r0 = (int)(rv - 1.f), r1 = (int)(rv + 3.f);
    const int w0 = (int)(wv - 1.f), w1 = (int)(wv + 3.f);
    for (int r = r0; r < r1; ++r) {
        if (!(-1 < r && r < rb)) continue;
        const double br = parzen((double)rv - r);
        const double rl = __ldg(&rlog[r]);
        for (int w = w0; w < w1; ++w) {
            if (!(-1 < w && w < fb)) continue;
            const double c = br * parzen_deriv((double)wv - w);
            sr = fma(c, rl, sr);
            sw = fma(c, __ldg(&wlog[w]), sw);
            sj = fma(c, __ldg(&logt[r + w * rb]), sj);
        }
    }
    return sr + sw - nmi * sj;
}

// ---------------------------------------------------------------------------------------------
// fused gradient: deformation + warp + spatial gradient + NMI voxel gradient
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(TILE_THREADS)
k_gradient(TileParams P, const float *__restrict__ ref, const float *__restrict__ flo,
           const int32_t *__restrict__ mask, const float *__restrict__ cpp,
           const double *__restrict__ logt, const nrb_objective *__restrict__ last,
           double weight, float *__restrict__ vgrad) {
    extern __shared__ float4 sm4[];
    float *sm = reinterpret_cast<float *>(sm4);
    const long long nv = (long long)P.nx * P.ny * P.nz;
    const double nmi = last->nmi;
    const double scale = weight / (last->entropy[2] * last->entropy[3]);
    const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
    for (int tile = blockIdx.x; tile < P.ntiles; tile += gridDim.x) {
        TileCtx T;
        tile_positions(P, cpp, tile, sm, T);
        const float *off = tile_offsets(P, sm);
        const int x = T.x0 + lx, y = T.y0 + ly;
        if (x >= P.nx || y >= P.ny) continue;  // no warp-collective operation below
        const int pre = pre_of(x, P.gsx);
        float bx[4];
        bspline_basis(frac_of(x, P.gsx, pre), bx);
        const int xo = pre - T.xa0;
#pragma unroll 1
        for (int zp = 0; zp < TILE_Z; ++zp) {
            const int z = T.z0 + zp;
            if (z >= P.nz) break;
            const long long idx = ((long long)z * P.ny + y) * P.nx + x;
            float out[3] = { 0.f, 0.f, 0.f };
            if (mask == nullptr || __ldg(&mask[idx]) > -1) {
                float wx, wy, wz, w, g[3];
                voxel_position(P, sm, off, ly, zp, xo, bx, wx, wy, wz);
                sample_floating<true>(flo, P.fnx, P.fny, P.fnz, P.flo_ijk, P.pad, wx, wy, wz, w, g);
                const float rv = __ldg(&ref[idx]);
                if (rv == rv && w == w) {
                    const double s = nmi_window(rv, w, logt, P.rb, P.fb, nmi);
#pragma unroll
                    for (int d = 0; d < 3; ++d) out[d] = (float)(scale * ((double)g[d] * s));
                }
            }
            vgrad[idx] = out[0];
            vgrad[nv + idx] = out[1];
            vgrad[2 * nv + idx] = out[2];
        }
    }
}

// ---------------------------------------------------------------------------------------------
// standalone Compute operations (same arithmetic, materialised intermediates)
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(TILE_THREADS)
k_deformation(TileParams P, const int32_t *__restrict__ mask, const float *__restrict__ cpp,
              float *__restrict__ def) {
    extern __shared__ float4 sm4[];
    float *sm = reinterpret_cast<float *>(sm4);
    const long long nv = (long long)P.nx * P.ny * P.nz;
    const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
    for (int tile = blockIdx.x; tile < P.ntiles; tile += gridDim.x) {
        TileCtx T;
        tile_positions(P, cpp, tile, sm, T);
        const float *off = tile_offsets(P, sm);
        const int x = T.x0 + lx, y = T.y0 + ly;
        if (x >= P.nx || y >= P.ny) continue;
        const int pre = pre_of(x, P.gsx);
        float bx[4];
        bspline_basis(frac_of(x, P.gsx, pre), bx);
        const int xo = pre - T.xa0;
        for (int zp = 0; zp < TILE_Z; ++zp) {
            const int z = T.z0 + zp;
            if (z >= P.nz) break;
            const long long idx = ((long long)z * P.ny + y) * P.nx + x;
            float wx = 0, wy = 0, wz = 0;
            if (mask == nullptr || __ldg(&mask[idx]) > -1) voxel_position(P, sm, off, ly, zp, xo, bx, wx, wy, wz);
            def[idx] = wx;
            def[nv + idx] = wy;
            def[2 * nv + idx] = wz;
        }
    }
}

template <bool kGrad>
__global__ void k_resample(long long nv, int fnx, int fny, int fnz, Mat34 M, float pad,
                           const float *__restrict__ flo, const float *__restrict__ def,
                           const int32_t *__restrict__ mask, float *__restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
         i += (long long)gridDim.x * blockDim.x) {
        const bool active = mask == nullptr || mask[i] > -1;
        if (!kGrad && !active) continue;
        float w = 0.f, g[3] = { 0.f, 0.f, 0.f };
        if (active)
            sample_floating<kGrad>(flo, fnx, fny, fnz, M, pad, def[i], def[nv + i], def[2 * nv + i], w, g);
        if (kGrad) {
            out[i] = g[0];
            out[nv + i] = g[1];
            out[2 * nv + i] = g[2];
        } else {
            out[i] = w;
        }
    }
}

__global__ void k_histogram(long long nv, int rb, int fb, const float *__restrict__ ref,
                            const float *__restrict__ war, const int32_t *__restrict__ mask,
                            uint32_t *__restrict__ ghist) {
    extern __shared__ uint32_t hs[];
    const int nbins = rb * fb;
    for (int i = threadIdx.x; i < nbins; i += blockDim.x) hs[i] = 0u;
    __syncthreads();
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long nround = (nv + stride - 1) / stride;
    for (long long k = 0; k < nround; ++k) {
        const long long i = k * stride + blockIdx.x * (long long)blockDim.x + threadIdx.x;
        int bin = -1;
        if (i < nv && (mask == nullptr || mask[i] > -1)) {
            const float r = ref[i], w = war[i];
            if (r == r && w == w && 0.f <= r && r < (float)rb && 0.f <= w && w < (float)fb)
                bin = (int)r + (int)w * rb;
        }
        const unsigned peers = __match_any_sync(0xffffffffu, bin);
        if (bin >= 0 && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&hs[bin], (uint32_t)__popc(peers));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nbins; i += blockDim.x) {
        const uint32_t v = hs[i];
        if (v) atomicAdd(&ghist[i], v);
    }
}

__global__ void k_nmi_voxel_gradient(long long nv, int rb, int fb, const float *__restrict__ ref,
                                     const float *__restrict__ war, const float *__restrict__ wgrad,
                                     const int32_t *__restrict__ mask, const double *__restrict__ logt,
                                     const nrb_objective *__restrict__ last, double weight,
                                     float *__restrict__ vgrad) {
    const double nmi = last->nmi;
    const double scale = weight / (last->entropy[2] * last->entropy[3]);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
         i += (long long)gridDim.x * blockDim.x) {
        if (mask != nullptr && mask[i] <= -1) continue;
        const float r = ref[i], w = war[i];
        if (!(r == r && w == w)) continue;
        const double s = nmi_window(r, w, logt, rb, fb, nmi);
        for (int d = 0; d < 3; ++d) {
            const float g = wgrad[d * nv + i];
            if (g == g) vgrad[d * nv + i] += (float)(scale * ((double)g * s));
        }
    }
}

// ---------------------------------------------------------------------------------------------
// histogram -> smoothed probabilities, FP64 entropies, log table (one block)
// ---------------------------------------------------------------------------------------------
constexpr int FIN_THREADS = 1024;

__device__ double block_sum(double v, double *red) {
    // fixed-shape tree: deterministic for a given block size
    const int tid = threadIdx.x;
    red[tid] = v;
    __syncthreads();
    for (int s = FIN_THREADS / 2; s > 0; s >>= 1) {
        if (tid < s) red[tid] += red[tid + s];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

// _reg_nmi.cpp:249-346 with the histogram as integer counts: 3-tap [1/6, float(2/3), 1/6]
// smoothing along the reference axis then the floating axis, normalisation by the total,
// marginals, entropies and the log table. The bending-energy partials of the same
// evaluation are summed here too, so one block produces the whole objective.
__global__ void __launch_bounds__(FIN_THREADS)
k_nmi_finalize(int rb, int fb, uint32_t *__restrict__ hist, double *__restrict__ pro,
               double *__restrict__ logt, nrb_objective *__restrict__ last,
               const double *__restrict__ be_partials, int n_be, double be_norm,
               double sim_weight, double be_weight, nrb_objective *__restrict__ obj) {
    __shared__ double red[FIN_THREADS];
    const int tid = threadIdx.x;
    const int nj = rb * fb, total = nj + rb + fb;
    const double k0 = parzen(-1.0), k1 = parzen(0.0);
    // smoothing along the reference axis into logt (scratch)
    for (int i = tid; i < nj; i += FIN_THREADS) {
        const int r = i % rb;
        double v = 0;
        if (r > 0) v += (double)hist[i - 1] * k0;
        v += (double)hist[i] * k1;
        if (r + 1 < rb) v += (double)hist[i + 1] * k0;
        logt[i] = v;
    }
    __syncthreads();
    double part = 0;
    for (int i = tid; i < total; i += FIN_THREADS) {
        double v = 0;
        if (i < nj) {
            const int f = i / rb;
            if (f > 0) v += logt[i - rb] * k0;
            v += logt[i] * k1;
            if (f + 1 < fb) v += logt[i + rb] * k0;
        }
        pro[i] = v;
        part += v;
    }
    const double mass = block_sum(part, red);  // syncs: pro complete, logt reads done
    for (int i = tid; i < nj; i += FIN_THREADS) {
        pro[i] /= mass;
        hist[i] = 0u;  // ready for the next evaluation
    }
    __syncthreads();
    // marginals, summed in the reference's sequential order
    for (int i = tid; i < rb + fb; i += FIN_THREADS) {
        double s = 0;
        if (i < rb) {
            for (int f = 0; f < fb; ++f) s += pro[i + rb * f];
        } else {
            const int f = i - rb;
            for (int r = 0; r < rb; ++r) s += pro[r + rb * f];
        }
        pro[nj + i] = s;
    }
    __syncthreads();
    double hr = 0, hw = 0, hj = 0;
    for (int i = tid; i < total; i += FIN_THREADS) {
        const double p = pro[i];
        double l = 0;
        if (p > 0) {
            l = log(p);
            if (i < nj) hj -= p * l;
            else if (i < nj + rb) hr -= p * l;
            else hw -= p * l;
        }
        logt[i] = l;
    }
    hr = block_sum(hr, red);
    hw = block_sum(hw, red);
    hj = block_sum(hj, red);
    double be = 0;
    for (int i = tid; i < n_be; i += FIN_THREADS) be += be_partials[i];
    be = block_sum(be, red) / be_norm;
    if (tid == 0) {
        nrb_objective o;
        // with a zero similarity weight the reference never evaluates the measure
        // (_reg_f3d.cpp:450-454): its weighted term is 0, not 0 * NaN
        o.nmi = sim_weight > 0 ? (hr + hw) / hj : 0.0;
        o.entropy[0] = hr;
        o.entropy[1] = hw;
        o.entropy[2] = hj;
        o.entropy[3] = mass;
        o.be = n_be > 0 ? be : 0.0;
        o.objective = (sim_weight > 0 ? sim_weight * o.nmi : 0.0) - (be_weight > 0 ? be_weight * o.be : 0.0);
        o.max_grad_len = last->max_grad_len;
        *last = o;
        if (obj) *obj = o;
    }
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
static TileParams make_tile_params(const nrb_workspace *ws, const nrb_geometry *g, float pad,
                                   int rb, int fb) {
    TileParams P{};
    P.nx = g->ref_dim[0];
    P.ny = g->ref_dim[1];
    P.nz = g->ref_dim[2];
    P.cx = g->cpp_dim[0];
    P.cy = g->cpp_dim[1];
    P.cz = g->cpp_dim[2];
    P.gsx = g->cpp_pixdim[0] / g->ref_pixdim[0];
    P.gsy = g->cpp_pixdim[1] / g->ref_pixdim[1];
    P.gsz = g->cpp_pixdim[2] / g->ref_pixdim[2];
    P.sa = ws->span[0];
    P.sb = ws->span[1];
    P.sc = ws->span[2];
    P.tiles_x = (P.nx + TILE_X - 1) / TILE_X;
    P.tiles_y = (P.ny + TILE_Y - 1) / TILE_Y;
    P.tiles_z = (P.nz + TILE_Z - 1) / TILE_Z;
    P.ntiles = P.tiles_x * P.tiles_y * P.tiles_z;
    P.fnx = g->flo_dim[0];
    P.fny = g->flo_dim[1];
    P.fnz = g->flo_dim[2];
    P.flo_ijk = to_mat34(g->flo_ijk);
    P.pad = pad;
    P.rb = rb;
    P.fb = fb;
    P.tile_floats = tile_smem_floats(P.sa, P.sb, P.sc);
    P.cnv = (long long)P.cx * P.cy * P.cz;
    return P;
}

template <typename K>
static nrb_status tile_grid(K kernel, size_t smem, int ntiles, int& grid) {
    static thread_local int configured_device = -1;
    int dev = 0;
    NRB_CUDA(cudaGetDevice(&dev));
    (void)configured_device;
    NRB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    int per_sm = 0;
    NRB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, TILE_THREADS, smem));
    if (per_sm < 1) return fail(NRB_ERR_UNSUPPORTED, "voxel tile does not fit in shared memory");
    grid = std::min(ntiles, per_sm * sm_count());
    return NRB_OK;
}

nrb_status launch_fused_objective(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g,
                                  const float *ref, const float *flo, const int32_t *mask,
                                  const float *cpp, float padding, cudaStream_t st) {
    const TileParams P = make_tile_params(ws, g, padding, nmi->rb, nmi->fb);
    const size_t smem = (size_t)P.tile_floats * 4 + (size_t)nmi->rb * nmi->fb * 4;
    int grid = 0;
    NRB_TRY(tile_grid(k_objective, smem, P.ntiles, grid));
    // algorithmic bytes: reference + floating (+ mask) per voxel, the grid once
    const double nv = (double)P.nx * P.ny * P.nz;
    const double bytes = nv * (mask ? 12.0 : 8.0) + 12.0 * (double)P.cnv;
    {
        KernelTimer timer(TK_OBJECTIVE, bytes, st);
        k_objective<<<grid, TILE_THREADS, smem, st>>>(P, ref, flo, mask, cpp, nmi->hist);
    }
    NRB_LAUNCHED("k_objective");
    return NRB_OK;
}

nrb_status launch_fused_gradient(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g,
                                 const float *ref, const float *flo, const int32_t *mask,
                                 const float *cpp, float padding, double weight, float *vgrad,
                                 cudaStream_t st) {
    const TileParams P = make_tile_params(ws, g, padding, nmi->rb, nmi->fb);
    const size_t smem = (size_t)P.tile_floats * 4;
    int grid = 0;
    NRB_TRY(tile_grid(k_gradient, smem, P.ntiles, grid));
    // algorithmic bytes: reference + floating (+ mask) read, voxel gradient written, grid once
    const double nv = (double)P.nx * P.ny * P.nz;
    const double bytes = nv * (mask ? 24.0 : 20.0) + 12.0 * (double)P.cnv;
    {
        KernelTimer timer(TK_GRADIENT, bytes, st);
        k_gradient<<<grid, TILE_THREADS, smem, st>>>(P, ref, flo, mask, cpp, nmi->logt, nmi->last, weight, vgrad);
    }
    NRB_LAUNCHED("k_gradient");
    return NRB_OK;
}

nrb_status launch_nmi_finalize(nrb_nmi *nmi, const double *be_partials, int n_be_partials,
                               int64_t cpp_nvox3, double sim_weight, double be_weight,
                               nrb_objective *obj, cudaStream_t st) {
    KernelTimer timer(TK_FINALIZE, (double)nmi->rb * nmi->fb * 4 + (double)nmi->total * 16, st);
    k_nmi_finalize<<<1, FIN_THREADS, 0, st>>>(nmi->rb, nmi->fb, nmi->hist, nmi->pro, nmi->logt, nmi->last,
                                               be_partials, n_be_partials, (double)cpp_nvox3, sim_weight,
                                               be_weight, obj);
    NRB_LAUNCHED("k_nmi_finalize");
    return NRB_OK;
}

}  // namespace nrb

using namespace nrb;

extern "C" nrb_status nrb_get_deformation_field(const nrb_geometry *g, const float *cpp,
                                                const int32_t *mask, float *def, void *stream) {
    if (!g || !cpp || !def) return fail(NRB_ERR_INVALID, "nrb_get_deformation_field: null pointer");
    nrb_workspace ws;
    NRB_TRY(validate_geometry(g));
    NRB_TRY(workspace_init(&ws, g));  // spans only; no allocation for this call
    const TileParams P = make_tile_params(&ws, g, 0.f, 0, 0);
    const size_t smem = (size_t)P.tile_floats * 4;
    int grid = 0;
    NRB_TRY(tile_grid(k_deformation, smem, P.ntiles, grid));
    k_deformation<<<grid, TILE_THREADS, smem, as_stream(stream)>>>(P, mask, cpp, def);
    NRB_LAUNCHED("k_deformation");
    return NRB_OK;
}

static nrb_status resample_common(const nrb_geometry *g, const float *flo, const float *def,
                                  const int32_t *mask, float pad, float *out, bool grad,
                                  void *stream) {
    if (!g || !flo || !def || !out) return fail(NRB_ERR_INVALID, "resample: null pointer");
    const long long nv = nvox(g->ref_dim);
    if (nv <= 0) return fail(NRB_ERR_INVALID, "resample: empty reference");
    const int threads = 256;
    const int grid = (int)std::min<long long>((nv + threads - 1) / threads, 8LL * sm_count() * 8);
    const Mat34 M = to_mat34(g->flo_ijk);
    if (grad)
        k_resample<true><<<grid, threads, 0, as_stream(stream)>>>(nv, g->flo_dim[0], g->flo_dim[1], g->flo_dim[2], M,
                                                                  pad, flo, def, mask, out);
    else
        k_resample<false><<<grid, threads, 0, as_stream(stream)>>>(nv, g->flo_dim[0], g->flo_dim[1], g->flo_dim[2], M,
                                                                   pad, flo, def, mask, out);
    NRB_LAUNCHED("k_resample");
    return NRB_OK;
}

extern "C" nrb_status nrb_resample_image(const nrb_geometry *g, const float *flo, const float *def,
                                         const int32_t *mask, float padding, float *warped,
                                         void *stream) {
    return resample_common(g, flo, def, mask, padding, warped, false, stream);
}

extern "C" nrb_status nrb_get_image_gradient(const nrb_geometry *g, const float *flo, const float *def,
                                             const int32_t *mask, float padding, float *grad,
                                             void *stream) {
    return resample_common(g, flo, def, mask, padding, grad, true, stream);
}

extern "C" nrb_status nrb_nmi_value(nrb_nmi *nmi, const nrb_geometry *g, const float *ref,
                                    const float *warped, const int32_t *mask, nrb_objective *obj,
                                    double *nmi_host, void *stream) {
    if (!nmi || !g || !ref || !warped) return fail(NRB_ERR_INVALID, "nrb_nmi_value: null pointer");
    const long long nv = nvox(g->ref_dim);
    cudaStream_t st = as_stream(stream);
    const int threads = 512;
    const int grid = (int)std::min<long long>((nv + threads - 1) / threads, 2LL * sm_count());
    const size_t smem = (size_t)nmi->rb * nmi->fb * 4;
    NRB_CUDA(cudaFuncSetAttribute(k_histogram, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    k_histogram<<<grid, threads, smem, st>>>(nv, nmi->rb, nmi->fb, ref, warped, mask, nmi->hist);
    NRB_LAUNCHED("k_histogram");
    NRB_TRY(launch_nmi_finalize(nmi, nullptr, 0, 1, 1.0, 0.0, obj, st));
    if (nmi_host) {
        nrb_objective o;
        NRB_CUDA(cudaMemcpyAsync(&o, nmi->last, sizeof(o), cudaMemcpyDeviceToHost, st));
        NRB_CUDA(cudaStreamSynchronize(st));
        *nmi_host = o.nmi;
    }
    return NRB_OK;
}

extern "C" nrb_status nrb_nmi_voxel_gradient(nrb_nmi *nmi, const nrb_geometry *g, const float *ref,
                                             const float *warped, const float *warped_grad,
                                             const int32_t *mask, double weight, float *vgrad,
                                             void *stream) {
    if (!nmi || !g || !ref || !warped || !warped_grad || !vgrad)
        return fail(NRB_ERR_INVALID, "nrb_nmi_voxel_gradient: null pointer");
    const long long nv = nvox(g->ref_dim);
    const int threads = 256;
    const int grid = (int)std::min<long long>((nv + threads - 1) / threads, 16LL * sm_count());
    k_nmi_voxel_gradient<<<grid, threads, 0, as_stream(stream)>>>(nv, nmi->rb, nmi->fb, ref, warped, warped_grad,
                                                                  mask, nmi->logt, nmi->last, weight, vgrad);
    NRB_LAUNCHED("k_nmi_voxel_gradient");
    return NRB_OK;
}
