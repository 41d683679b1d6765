// Voxel-pass kernels of the F3D objective and gradient.
//
// Work item: a column of 32 (x) by ty (y) reference voxels over a chunk of z slices. The block
// stages the control points the item depends on in shared memory once (batched loads),
// together with the z basis of every slice of the chunk; then every thread walks its own voxel
// column along z. The cubic B-spline sum sum_{a,b,c} Bx_a By_b Bz_c CP is evaluated
// separably: for each node plane k the thread contracts the 4x4 (a, b) neighbourhood with its
// fixed x/y weights into S(k) (20 FMAs per component), keeps a rolling window of the four planes
// the current slice needs, and contracts z with 4 FMAs per component. z is uniform across the
// block, so the window shifts without divergence and the walk needs no barrier.
//
// The deformation field never leaves the SM in the fused kernels: it is consumed at once by the
// trilinear warp and then by the joint histogram (objective) or by the spatial gradient and the
// NMI voxel gradient (gradient). Blocks are persistent; in the objective kernel each keeps a
// shared-memory joint histogram and flushes it with one atomic per non-zero bin.
#include <cooperative_groups.h>
#include <cuda_pipeline.h>

#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "nrb_state.cuh"

namespace cg = cooperative_groups;

namespace nrb {

__device__ __forceinline__ int pre_of(int v, float gs) { return (int)((float)v / gs); }

__device__ __forceinline__ float frac_of(int v, float gs, int pre) {
    const float t = (float)v / gs - (float)pre;
    return t < 0.f ? 0.f : t;
}

// shared floats of the per-item tables: z basis [zchunk][4], z node index [zchunk] and the
// identity z position of each slice as a (hi, lo) float pair [zchunk][2]
__host__ __device__ inline int walk_table_floats(int zchunk) { return 7 * zchunk; }

// Positions as identity + displacement. With the grid's voxel -> mm matrix free of off-diagonal
// terms, the identity position of node k along axis c is io[c] + is[c] * k, and the cubic
// B-spline reproduces linear functions exactly, so for a voxel at grid coordinate pre + t
// (pre = node index, t = basis fraction)
//     sum_k B_k(t) CP_k = io + is * (pre + 1 + t) + sum_k B_k(t) (CP_k - io - is * k).
// The walk sums the displacements CP_k - (io + is * k) in float (magnitudes of a few mm, so their
// rounding errors are ~1e-7 mm) and adds the identity part, evaluated in double and held as a
// (hi, lo) float pair, at the end: the position is then within about one float ulp of the FP64
// evaluation of the same sum, where summing absolute positions (hundreds of mm) in float drifts
// by several ulps. With a general grid matrix io = is = 0 and the sum is the absolute one.
__device__ __forceinline__ double identity_coord(float io, float is, int pre, double t) {
    return (double)io + (double)is * ((double)(pre + 1) + t);
}

__device__ __forceinline__ void split_hi_lo(double v, float& hi, float& lo) {
    hi = (float)v;
    lo = (float)(v - (double)hi);
}

// basis fraction of voxel v in double (the FP64 evaluation's t), clamped as frac_of clamps
__device__ __forceinline__ double frac_of_d(int v, float gs, int pre) {
    const double t = (double)v / (double)gs - (double)pre;
    return t < 0.0 ? 0.0 : t;
}

struct Item {
    int x0, y0, z0, z1, xa0, yb0, zc0;
};

// Stages the control points of `item` into cp[3][sc][sb][sa] and the z basis of each slice into
// the tables. The values are staged as they are (not relative to the item), so a voxel's
// position is the same float whatever the item decomposition, and so are the results.
// With kTrial the control points are the line search's trial values best + scale * grad
// (`cpp` = best), formed here instead of in a separate update pass. Called by every thread of
// the block.
template <bool kTrial = false>
__device__ __forceinline__ void stage_item(const WalkParams& P, const float *__restrict__ cpp, int item,
                                           float *cp, float *zb, int *zk, float2 *zid, Item& I,
                                           const float *__restrict__ grad = nullptr, float scale = 0.f) {
    const int tx = item % P.tiles_x;
    const int rest = item / P.tiles_x;
    const int ty = rest % P.tiles_y;
    const int tz = rest / P.tiles_y;
    I.x0 = tx * COL_X;
    I.y0 = ty * P.ty;
    I.z0 = tz * P.zchunk;
    I.z1 = min(I.z0 + P.zchunk, P.nz);
    I.xa0 = pre_of(I.x0, P.gsx);
    I.yb0 = pre_of(I.y0, P.gsy);
    I.zc0 = pre_of(I.z0, P.gsz);
    const int na = pre_of(min(I.x0 + COL_X - 1, P.nx - 1), P.gsx) + 4 - I.xa0;
    const int nb = pre_of(min(I.y0 + P.ty - 1, P.ny - 1), P.gsy) + 4 - I.yb0;
    const int nc = pre_of(I.z1 - 1, P.gsz) + 4 - I.zc0;
    const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
    __syncthreads();  // the previous item's readers are done
    // one pass: the node planes of one (component, row, column) are independent loads, batched
    // four at a time so their latencies overlap
    const int gplane = P.cx * P.cy, splane = P.sb * P.sa;
#pragma unroll
    for (int c = 0; c < 3; ++c)
        for (int jb = ly; jb < nb; jb += P.ty)
            for (int ia = lx; ia < na; ia += 32) {
                const int src = c * P.cnv + (I.zc0 * P.cy + I.yb0 + jb) * P.cx + I.xa0 + ia;
                float *dst = cp + (c * P.sc * P.sb + jb) * P.sa + ia;
                const float *g = kTrial ? grad : nullptr;
                // the identity position of this node row (component c varies along axis c only)
                const double io = (double)P.io[c], is = (double)P.is[c];
                const double rowid = c == 0 ? io + is * (double)(I.xa0 + ia)
                                   : c == 1 ? io + is * (double)(I.yb0 + jb) : io + is * (double)I.zc0;
                const double kstep = c == 2 ? is : 0.0;
                int kc = 0;
                for (; kc + 4 <= nc; kc += 4) {
                    const float v0 = trial_cp(cpp, g, scale, src + kc * gplane);
                    const float v1 = trial_cp(cpp, g, scale, src + (kc + 1) * gplane);
                    const float v2 = trial_cp(cpp, g, scale, src + (kc + 2) * gplane);
                    const float v3 = trial_cp(cpp, g, scale, src + (kc + 3) * gplane);
                    dst[kc * splane] = (float)((double)v0 - (rowid + kstep * kc));
                    dst[(kc + 1) * splane] = (float)((double)v1 - (rowid + kstep * (kc + 1)));
                    dst[(kc + 2) * splane] = (float)((double)v2 - (rowid + kstep * (kc + 2)));
                    dst[(kc + 3) * splane] = (float)((double)v3 - (rowid + kstep * (kc + 3)));
                }
                for (; kc < nc; ++kc)
                    dst[kc * splane] = (float)((double)trial_cp(cpp, g, scale, src + kc * gplane) - (rowid + kstep * kc));
            }
    for (int zi = threadIdx.x; zi < I.z1 - I.z0; zi += blockDim.x) {
        const int z = I.z0 + zi;
        const int pz = pre_of(z, P.gsz);
        zk[zi] = pz - I.zc0;
        bspline_basis(frac_of(z, P.gsz, pz), zb + 4 * zi);
        float2 h;
        split_hi_lo(identity_coord(P.io[2], P.is[2], pz, frac_of_d(z, P.gsz, pz)), h.x, h.y);
        zid[zi] = h;
    }
    __syncthreads();
}

// Per-thread walker: x/y weights of the thread's column and the rolling window of the four
// node planes contracted over (a, b).
struct Column {
    int x, y;
    bool inside;     // the column lies inside the reference volume
    float bx[4], by[4];
    int xoff, yrow;  // first node of the column relative to the staged block (x, y)
    const float *base;
    int win;         // relative z node index of S[0]
    float S[4][3];
    float hx, lx, hy, ly;  // identity x and y positions of the column as (hi, lo) float pairs
};

__device__ __forceinline__ void column_init(const WalkParams& P, const Item& I, const float *cp, Column& C) {
    const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
    C.x = I.x0 + lx;
    C.y = I.y0 + ly;
    C.inside = C.x < P.nx && C.y < P.ny;
    const int xc = min(C.x, P.nx - 1), yc = min(C.y, P.ny - 1);
    const int px = pre_of(xc, P.gsx), py = pre_of(yc, P.gsy);
    bspline_basis(frac_of(xc, P.gsx, px), C.bx);
    bspline_basis(frac_of(yc, P.gsy, py), C.by);
    split_hi_lo(identity_coord(P.io[0], P.is[0], px, frac_of_d(xc, P.gsx, px)), C.hx, C.lx);
    split_hi_lo(identity_coord(P.io[1], P.is[1], py, frac_of_d(yc, P.gsy, py)), C.hy, C.ly);
    C.xoff = px - I.xa0;
    C.yrow = py - I.yb0;
    C.base = cp + C.yrow * P.sa + C.xoff;
    C.win = INT_MIN;
}

// S for relative node plane k
__device__ __forceinline__ void column_plane(const WalkParams& P, const Column& C, int k, float out[3]) {
    const int cs = P.sc * P.sb * P.sa;
    const float *p = C.base + k * P.sb * P.sa;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float *q = p + c * cs;
        float s = 0.f;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const float *r = q + b * P.sa;
            float t = C.bx[0] * r[0];
            t = fmaf(C.bx[1], r[1], t);
            t = fmaf(C.bx[2], r[2], t);
            t = fmaf(C.bx[3], r[3], t);
            s = fmaf(C.by[b], t, s);
        }
        out[c] = s;
    }
}

// The x contraction of every (component, node plane, node row) of the item for the 32 columns
// of its x tile, X[c][k][b][lane] = sum_a bx_lane[a] cp[c][k][b][px_lane - xa0 + a], built once
// per item by the whole block (same operations, same order as column_plane's inner sum). Walks
// then contract only over the 4 rows: 4 shared loads and 4 FMAs per component and plane instead
// of 16 + 16. Called by every thread after stage_item; ends with a barrier.
__device__ __forceinline__ void build_xrows(const WalkParams& P, const Column& C, const float *cp, float *X) {
    const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
    const int rows = 3 * P.sc * P.sb;  // (c, k, b) rows of the staged block, b fastest
    for (int e = ly; e < rows; e += P.ty) {
        const float *r = cp + e * P.sa + C.xoff;
        float t = C.bx[0] * r[0];
        t = fmaf(C.bx[1], r[1], t);
        t = fmaf(C.bx[2], r[2], t);
        t = fmaf(C.bx[3], r[3], t);
        X[e * 32 + lx] = t;
    }
    __syncthreads();
}

// S for relative node plane k from the x-contracted rows
__device__ __forceinline__ void column_plane_x(const WalkParams& P, const Column& C, const float *X, int k,
                                               float out[3]) {
    const int lx = threadIdx.x & 31;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float *q = X + ((c * P.sc + k) * P.sb + C.yrow) * 32 + lx;
        float s = 0.f;
#pragma unroll
        for (int b = 0; b < 4; ++b) s = fmaf(C.by[b], q[b * 32], s);
        out[c] = s;
    }
}

// World position (mm) of slice index zi (relative to the item) of the thread's column; zi must
// not decrease between calls. X: the item's x-contracted rows, or null.
__device__ __forceinline__ void column_position(const WalkParams& P, const Item& I, Column& C, const float *zb,
                                                const int *zk, const float2 *zid, int zi, float pos[3],
                                                const float *X = nullptr) {
    const int pz = zk[zi];
    if (pz != C.win) {
        if (pz == C.win + 1) {
#pragma unroll
            for (int t = 0; t < 3; ++t)
#pragma unroll
                for (int c = 0; c < 3; ++c) C.S[t][c] = C.S[t + 1][c];
            if (X) column_plane_x(P, C, X, pz + 3, C.S[3]);
            else column_plane(P, C, pz + 3, C.S[3]);
        } else {
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                if (X) column_plane_x(P, C, X, pz + t, C.S[t]);
                else column_plane(P, C, pz + t, C.S[t]);
            }
        }
        C.win = pz;
    }
    const float4 bz = reinterpret_cast<const float4 *>(zb)[zi];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float s = bz.x * C.S[0][c];
        s = fmaf(bz.y, C.S[1][c], s);
        s = fmaf(bz.z, C.S[2][c], s);
        s = fmaf(bz.w, C.S[3][c], s);
        pos[c] = s;
    }
    // identity part: hi + (lo + displacement), two roundings on values far below an ulp of hi
    const float2 hz = zid[zi];
    pos[0] = __fadd_rn(C.hx, __fadd_rn(C.lx, pos[0]));
    pos[1] = __fadd_rn(C.hy, __fadd_rn(C.ly, pos[1]));
    pos[2] = __fadd_rn(hz.x, __fadd_rn(hz.y, pos[2]));
}

// mm -> floating voxel as Mat44Mul does it (reg-lib/cpu/Maths.hpp:272-286): the products of
// two floats are exact in double, so one rounding to double and one to float. With no
// off-diagonal terms the single-precision FMA rounds the same exact value once instead of twice
// (the two agree except when the exact value falls within 2^-53 of a float rounding boundary)
// and keeps the conversions off the XU pipe.
// kDiag: 1 = M has no off-diagonal terms, 0 = general M, -1 = decided by `diag` at run time
template <int kDiag>
__device__ __forceinline__ void to_floating_voxel(const Mat34& M, int diag, float x, float y, float z,
                                                  float& fx, float& fy, float& fz) {
    if (kDiag == 1 || (kDiag < 0 && diag)) {
        fx = __fmaf_rn(M.m[0], x, M.m[3]);
        fy = __fmaf_rn(M.m[5], y, M.m[7]);
        fz = __fmaf_rn(M.m[10], z, M.m[11]);
        return;
    }
    const double dx = x, dy = y, dz = z;
    fx = (float)((double)M.m[0] * dx + (double)M.m[1] * dy + (double)M.m[2] * dz + (double)M.m[3]);
    fy = (float)((double)M.m[4] * dx + (double)M.m[5] * dy + (double)M.m[6] * dz + (double)M.m[7]);
    fz = (float)((double)M.m[8] * dx + (double)M.m[9] * dy + (double)M.m[10] * dz + (double)M.m[11]);
}

// floor(v) as float and as int. v is clamped to +-2^21 first: every position that far out lies
// outside any volume this library accepts, and the clamp keeps px + 1 from overflowing.
__device__ __forceinline__ int floor_split(float v, float& fl) {
    v = fminf(fmaxf(v, -2097152.0f), 2097152.0f);
    fl = floorf(v);
    return __float2int_rd(v);
}

// (int)v for 0 <= v (truncation == floor there)
__device__ __forceinline__ int trunc_nonneg(float v) { return __float2int_rz(v); }

// Trilinear sample of the floating image at world position (x, y, z) with the padding rule of
// ResampleImage3D (an out-of-volume tap contributes padding * weight, so NaN padding poisons a
// border voxel even through a zero weight) and, when kGrad, the spatial derivative of
// TrilinearImageGradient (NaN components -> 0).
//
// Layout: `flo` points at voxel (0, 0, 0), rows are `sy` and slices `sz` floats apart, and
// `margin` voxels holding the padding value surround the volume on every side (0: a dense
// volume). Warps whose 32 samples have all eight taps inside the volume or its margin take the
// plain 8-load path: a tap in the margin reads the padding value from memory, the very value
// the clamped path substitutes, so the two paths give the same numbers. Other warps read
// clamped in-volume addresses and select the padding value for out-of-volume taps, with no
// divergence.
// The 2x2 footprint of layer `layer` whose lower corner is texel (x0, y0), from one texture
// gather (tld4) of a 2D layered float array at (x0 + 1, y0 + 1): the texels come back as stored.
// The gather returns (x0, y0 + 1), (x0 + 1, y0 + 1), (x0 + 1, y0), (x0, y0) in that order;
// v[b][a] = texel (x0 + a, y0 + b).
__device__ __forceinline__ void gather_footprint(unsigned long long tex, int layer, float x0p1, float y0p1,
                                                 float v[2][2]) {
    float r0, r1, r2, r3;
    asm("tld4.r.a2d.v4.f32.f32 {%0, %1, %2, %3}, [%4, {%5, %6, %7, %8}];"
        : "=f"(r0), "=f"(r1), "=f"(r2), "=f"(r3)
        : "l"(tex), "r"(layer), "f"(x0p1), "f"(y0p1), "f"(0.f));
    v[1][0] = r0;
    v[1][1] = r1;
    v[0][1] = r2;
    v[0][0] = r3;
}

// tex (optional; needs margin >= 2): the same floating image with its margin as a 2D layered
// float array (layer k = slice k - margin, texel (i, j) = voxel (i - margin, j - margin)); every
// sample then fetches each slice's 2x2 footprint with one gather instead of four loads, with no
// warp vote and no clamped path.
template <bool kGrad, int kDiag = -1>
__device__ __forceinline__ void sample_floating(const float *__restrict__ flo, unsigned long long tex, int fnx, int fny,
                                                int fnz, int sy, int sz, int margin, const Mat34& M,
                                                int diag, float pad, float x, float y, float z,
                                                float& val, float g[3]) {
    float fx, fy, fz;
    to_floating_voxel<kDiag>(M, diag, x, y, z, fx, fy, fz);
    float flx, fly, flz;
    const int px = floor_split(fx, flx), py = floor_split(fy, fly), pz = floor_split(fz, flz);
    const float rx = fx - flx, ry = fy - fly, rz = fz - flz;
    const float bx0 = 1.f - rx, by0 = 1.f - ry, bz0 = 1.f - rz;
    float v[2][2][2];
    // -margin <= p and p + 1 <= n - 1 + margin on every axis (|p| <= 2^21: no overflow)
    const bool plain = (unsigned)(px + margin) < (unsigned)(fnx + 2 * margin - 1) &&
                       (unsigned)(py + margin) < (unsigned)(fny + 2 * margin - 1) &&
                       (unsigned)(pz + margin) < (unsigned)(fnz + 2 * margin - 1);
    if (tex) {
        // every sample, no vote: the footprint's first texel (p + margin on each axis) clamped to
        // [0, n + 2 margin - 2]. Unclamped, that is the plain path's footprint; clamped, both taps
        // on that axis lie outside the volume (p < -margin or p > n + margin - 2) and the clamped
        // footprint lies in the margin (margin >= 2), so they read the padding value, as the
        // clamped path substitutes it. Texels past the padded extent are never read.
        const float off = (float)(margin + 1);
        const float tx = fminf(fmaxf(flx + off, 1.f), (float)(fnx + 2 * margin - 1));
        const float ty = fminf(fmaxf(fly + off, 1.f), (float)(fny + 2 * margin - 1));
        const int layer = min(max(pz + margin, 0), fnz + 2 * margin - 2);
        gather_footprint(tex, layer, tx, ty, v[0]);
        gather_footprint(tex, layer + 1, tx, ty, v[1]);
    } else if (__all_sync(__activemask(), plain)) {
        const float *p = flo + (pz * sz + py * sy + px);
        v[0][0][0] = __ldg(p);
        v[0][0][1] = __ldg(p + 1);
        v[0][1][0] = __ldg(p + sy);
        v[0][1][1] = __ldg(p + sy + 1);
        v[1][0][0] = __ldg(p + sz);
        v[1][0][1] = __ldg(p + sz + 1);
        v[1][1][0] = __ldg(p + sz + sy);
        v[1][1][1] = __ldg(p + sz + sy + 1);
    } else {
        const bool inx[2] = { (unsigned)px < (unsigned)fnx, (unsigned)(px + 1) < (unsigned)fnx };
        const bool iny[2] = { (unsigned)py < (unsigned)fny, (unsigned)(py + 1) < (unsigned)fny };
        const bool inz[2] = { (unsigned)pz < (unsigned)fnz, (unsigned)(pz + 1) < (unsigned)fnz };
        const int cx[2] = { min(max(px, 0), fnx - 1), min(max(px + 1, 0), fnx - 1) };
        const int cy[2] = { min(max(py, 0), fny - 1), min(max(py + 1, 0), fny - 1) };
        const int cz[2] = { min(max(pz, 0), fnz - 1), min(max(pz + 1, 0), fnz - 1) };
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const float *row = flo + cz[c] * sz + cy[b] * sy;
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    const float t = __ldg(row + cx[a]);
                    v[c][b][a] = (inx[a] && iny[b] && inz[c]) ? t : pad;
                }
            }
    }
    const float yv0 = fmaf(v[0][0][1], rx, v[0][0][0] * bx0);
    const float yv1 = fmaf(v[0][1][1], rx, v[0][1][0] * bx0);
    const float zv0 = fmaf(yv1, ry, yv0 * by0);
    const float yw0 = fmaf(v[1][0][1], rx, v[1][0][0] * bx0);
    const float yw1 = fmaf(v[1][1][1], rx, v[1][1][0] * bx0);
    const float zv1 = fmaf(yw1, ry, yw0 * by0);
    val = fmaf(zv1, rz, zv0 * bz0);
    if (kGrad) {
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

constexpr int WALK_GROUP = 1;  // slices per step of the walk (two in flight measured 2% slower)

// shared-memory layout of a walk block: cp block | z basis | z node index | kernel-specific
struct WalkSmem {
    float *cp, *zb;
    int *zk;
    float2 *zid;
    char *tail;
};

__device__ __forceinline__ WalkSmem walk_smem(const WalkParams& P, void *base) {
    WalkSmem s;
    s.cp = reinterpret_cast<float *>(base);
    s.zb = s.cp + ((3 * P.sc * P.sb * P.sa + 3) & ~3);  // 16-byte aligned rows of 4 basis values
    s.zid = reinterpret_cast<float2 *>(s.zb + 4 * P.zchunk);  // 8-byte aligned pairs
    s.zk = reinterpret_cast<int *>(s.zid + P.zchunk);
    s.tail = reinterpret_cast<char *>(s.zk + P.zchunk);
    // 16-byte alignment of the tail
    s.tail = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(s.tail) + 15) & ~uintptr_t(15));
    return s;
}

size_t walk_smem_bytes(const WalkPlan& W) {
    return ((size_t)W.cp_floats + 4 + (size_t)walk_table_floats(W.zchunk)) * 4 + 16;
}

// ---------------------------------------------------------------------------------------------
// fused objective: deformation + warp + joint histogram
// ---------------------------------------------------------------------------------------------
// Shared histogram of a walk block: zeroed four bins at a time (it starts 16-byte aligned) and
// flushed with one global atomic per non-zero bin (merging the blocks of a cluster through
// distributed shared memory first was measured slower at every volume size). flush_hist starts
// with a barrier (every count of the block is in).
__device__ __forceinline__ void zero_hist(uint32_t *h, int nbins) {
    for (int i = threadIdx.x; i < (nbins + 3) / 4; i += blockDim.x) reinterpret_cast<uint4 *>(h)[i] = make_uint4(0, 0, 0, 0);
}

__device__ __forceinline__ void flush_hist(const uint32_t *h, int nbins, uint32_t *__restrict__ ghist) {
    __syncthreads();
    for (int i = threadIdx.x; i < nbins / 4; i += blockDim.x) {
        const uint4 c = reinterpret_cast<const uint4 *>(h)[i];
        if (c.x) atomicAdd(&ghist[4 * i], c.x);
        if (c.y) atomicAdd(&ghist[4 * i + 1], c.y);
        if (c.z) atomicAdd(&ghist[4 * i + 2], c.z);
        if (c.w) atomicAdd(&ghist[4 * i + 3], c.w);
    }
    for (int i = (nbins & ~3) + (int)threadIdx.x; i < nbins; i += blockDim.x) {
        const uint32_t c = h[i];
        if (c) atomicAdd(&ghist[i], c);
    }
}

// One item of the fused objective (deformation + warp + joint histogram): stage the item's
// control points (the trial values best - len * grad when grad is given), walk its columns and
// count every active voxel's (reference, warped) bin pair into the block's histogram h. Called
// by every thread of the block.
template <bool kXs, bool kDiag>
__device__ __forceinline__ void objective_item(const WalkParams& P, const WalkSmem& S, uint32_t *h, float *X,
                                               int item, const float *__restrict__ ref,
                                               const float *__restrict__ flo, const int32_t *__restrict__ mask,
                                               const float *__restrict__ cpp, const float *__restrict__ grad,
                                               float scale) {
    const int lane = threadIdx.x & 31;
    const float frb = (float)P.rb, ffb = (float)P.fb;
    Item I;
    stage_item<true>(P, cpp, item, S.cp, S.zb, S.zk, S.zid, I, grad, scale);
    Column C;
    column_init(P, I, S.cp, C);
    if (kXs) build_xrows(P, C, S.cp, X);
    const int nzi = I.z1 - I.z0;
    int idx = (I.z0 * P.ny + C.y) * P.nx + C.x;
    const int zstride = P.nx * P.ny;
    for (int zi = 0; zi < nzi; zi += WALK_GROUP) {
        int bin[WALK_GROUP];
#pragma unroll
        for (int u = 0; u < WALK_GROUP; ++u) {
            const int zu = min(zi + u, nzi - 1);
            float pos[3];
            column_position(P, I, C, S.zb, S.zk, S.zid, zu, pos, kXs ? X : nullptr);
            bin[u] = -1;
            if (C.inside && zi + u < nzi) {
                const int vi = idx + u * zstride;
                if (mask == nullptr || __ldg(&mask[vi]) > -1) {
                    float w, g[3];
                    sample_floating<false, kDiag ? 1 : 0>(flo, P.ftex, P.fnx, P.fny, P.fnz, P.fsy, P.fsz, P.fmargin,
                                                          P.flo_ijk, P.flo_diag, P.pad, pos[0], pos[1], pos[2], w, g);
                    const float rv = __ldg(&ref[vi]);
                    if (0.f <= rv && rv < frb && 0.f <= w && w < ffb)  // false for NaN
                        bin[u] = trunc_nonneg(rv) + trunc_nonneg(w) * P.rb;
                }
            }
        }
        idx += WALK_GROUP * zstride;
#pragma unroll
        for (int u = 0; u < WALK_GROUP; ++u) {
            // a warp whose 32 voxels share one bin (background) adds 32 with one atomic
            const int b0 = __shfl_sync(0xffffffffu, bin[u], 0);
            if (__all_sync(0xffffffffu, bin[u] == b0)) {
                if (lane == 0 && b0 >= 0) atomicAdd(&h[b0], 32u);
            } else if (bin[u] >= 0) {
                atomicAdd(&h[bin[u]], 1u);
            }
        }
    }
}

// shared layout of an objective block: walk | histogram | x-contracted rows (P.xs)
__device__ __forceinline__ void objective_smem(const WalkParams& P, void *base, WalkSmem& S, uint32_t *&h, float *&X) {
    S = walk_smem(P, base);
    h = reinterpret_cast<uint32_t *>(S.tail);
    X = reinterpret_cast<float *>(h + ((P.rb * P.fb + 3) & ~3));
}

// ---------------------------------------------------------------------------------------------
// fused objective: deformation + warp + joint histogram
// ---------------------------------------------------------------------------------------------
// kXs: the item's x-contracted node rows are staged in shared memory; kDiag: the floating
// image's mm -> voxel matrix has no off-diagonal terms (launch-time choices made template
// parameters, so the walk carries no test for them)
template <bool kTrial, bool kXs, bool kDiag>
__global__ void __launch_bounds__(32 * TY_OBJECTIVE, 2)
k_objective(WalkParams P, const float *__restrict__ ref, const float *__restrict__ flo,
            const int32_t *__restrict__ mask, const float *__restrict__ cpp,
            uint32_t *__restrict__ ghist, const float *__restrict__ grad, const OptState *__restrict__ step) {
    extern __shared__ float4 sm4[];
    WalkSmem S;
    uint32_t *h;
    float *X;
    objective_smem(P, sm4, S, h, X);
    const int nbins = P.rb * P.fb;
    zero_hist(h, nbins);
    if (kTrial) pdl_wait();  // the trial position and step length come from the previous launch
    pdl_launch_dependents();  // the finalize may start its preamble (it waits for the counts)
    const float scale = kTrial ? -step->cur_len : 0.f;
    for (int item = blockIdx.x; item < P.nitems; item += gridDim.x)
        objective_item<kXs, kDiag>(P, S, h, X, item, ref, flo, mask, cpp, kTrial ? grad : nullptr, scale);
    flush_hist(h, nbins, ghist);
}

// Sum over the 4x4 Parzen window of reg_getVoxelBasedNmiGradient3d (_reg_nmi.cpp:548-571):
// returns refDeriv + warDeriv - nmi * jointDeriv for a unit spatial gradient. The window's
// basis values are evaluated once (4 + 4), then its 16 (r, w) pairs are summed in the
// reference's r-major order.
__device__ __forceinline__ double nmi_window(float rv, float wv, const double *logt, int rb, int fb, double nmi) {
    const double *rlog = logt + rb * fb;
    const double *wlog = rlog + rb;
    const int r0 = (int)(rv - 1.f), r1 = (int)(rv + 3.f);
    const int w0 = (int)(wv - 1.f), w1 = (int)(wv + 3.f);
    double br[4], dw[4], wl[4];
    int wok[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int r = r0 + t, w = w0 + t;
        const bool rok = r < r1 && -1 < r && r < rb;
        br[t] = rok ? parzen((double)rv - r) : 0.0;
        wok[t] = w < w1 && -1 < w && w < fb;
        dw[t] = wok[t] ? parzen_deriv((double)wv - w) : 0.0;
        wl[t] = wok[t] ? wlog[w] : 0.0;
    }
    double sr = 0, sw = 0, sj = 0;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int r = r0 + t;
        if (!(r < r1 && -1 < r && r < rb)) continue;
        const double rl = rlog[r];
        const double *jrow = logt + r;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (!wok[u]) continue;
            const double c = br[t] * dw[u];
            sr = fma(c, rl, sr);
            sw = fma(c, wl[u], sw);
            sj = fma(c, jrow[(w0 + u) * rb], sj);
        }
    }
    return sr + sw - nmi * sj;
}

// The same window in FP32 on an FP32 copy of the log table (the fused gradient pass): the
// per-voxel terms are a 16-tap weighted sum whose FP32 rounding (~1e-6 relative) stays far
// below the voxel-face jumps of the trilinear spatial gradient, while the FP64 normalisation
// constant (weight / (H_joint * total)) multiplies it afterwards.
__device__ __forceinline__ float nmi_window_f(float rv, float wv, const float *logt, int rb, int fb, float nmi) {
    const float *rlog = logt + rb * fb;
    const float *wlog = rlog + rb;
    const int r0 = (int)(rv - 1.f), r1 = (int)(rv + 3.f);
    const int w0 = (int)(wv - 1.f), w1 = (int)(wv + 3.f);
    // taps outside the window or the table get weight 0 and a clamped (valid) table index, so
    // the sums need no branches; the marginal terms factor out of the double sum:
    //   sum_tu br_t dw_u rlog_t = (sum_t br_t rlog_t)(sum_u dw_u), and likewise for wlog
    float br[4], dw[4], rl[4], wl[4];
    int ri[4], wi[4];
    if (rv >= 1.f && wv >= 1.f && rv < (float)(rb - 2) && wv < (float)(fb - 2)) {
        // r0 + 1 = floor(rv): the four taps sit at rv - r = f + 1, f, f - 1, f - 2 (all exact)
        // with f the fractional part, each inside one known piece of the kernel. The pieces
        // parzenf / parzen_derivf would select are written out with their operations in their
        // order (sign changes are exact), so every value is the same float; only |x| = 1 at
        // f = 0 falls in the other piece and is given its value (1/6) explicitly.
        const float f = rv - (float)(r0 + 1), mf = 1.f - f;
        br[0] = mf * mf * mf * (1.f / 6.f);
        br[1] = (2.0f / 3.0f) + (0.5f * f - 1.f) * f * f;
        br[2] = mf < 1.f ? (2.0f / 3.0f) + (0.5f * mf - 1.f) * mf * mf : (1.f / 6.f);
        br[3] = f * f * f * (1.f / 6.f);
        const float g = wv - (float)(w0 + 1), mg = 1.f - g;
        dw[0] = -0.5f * mg * mg;
        dw[1] = (1.5f * g - 2.f) * g;
        dw[2] = (1.5f * mg - 2.f) * -mg;
        dw[3] = 0.5f * g * g;
        // 1 <= rv < rb - 2: the taps r0 .. r0 + 3 = floor(rv) - 1 .. floor(rv) + 2 all lie in the
        // table (and likewise for wv), so none is masked or clamped
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            ri[t] = r0 + t;
            wi[t] = (w0 + t) * rb;
            rl[t] = rlog[r0 + t];
            wl[t] = wlog[w0 + t];
        }
    } else {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int r = r0 + t, w = w0 + t;
            const bool rok = r < r1 && -1 < r && r < rb;
            const bool wok = w < w1 && -1 < w && w < fb;
            ri[t] = min(max(r, 0), rb - 1);
            wi[t] = min(max(w, 0), fb - 1) * rb;
            br[t] = rok ? parzenf(rv - (float)r) : 0.f;
            dw[t] = wok ? parzen_derivf(wv - (float)w) : 0.f;
            rl[t] = rlog[ri[t]];
            wl[t] = wlog[min(max(w, 0), fb - 1)];
        }
    }
    float sbr = 0.f, sdw = 0.f, sr = 0.f, sw = 0.f, sj = 0.f;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        sbr += br[t];
        sdw += dw[t];
        sr = fmaf(br[t], rl[t], sr);
        sw = fmaf(dw[t], wl[t], sw);
        float row = 0.f;
#pragma unroll
        for (int u = 0; u < 4; ++u) row = fmaf(dw[u], logt[ri[t] + wi[u]], row);
        sj = fmaf(br[t], row, sj);
    }
    return fmaf(sr, sdw, sbr * sw) - nmi * sj;
}

// ---------------------------------------------------------------------------------------------
// fused gradient: deformation + warp + spatial gradient + NMI voxel gradient
// ---------------------------------------------------------------------------------------------
// The NMI quantities one gradient evaluation reads: the log table of the best position's table
// set, its NMI and the normalisation weight / (H_joint * total).
struct GradientTables {
    const double *logt;
    double nmi, scale;
    float nmi_f, scale_f;
};

__device__ __forceinline__ GradientTables gradient_tables(const double *logt0, const nrb_objective *last0,
                                                          const double *logt1, const nrb_objective *last1,
                                                          bool second, double weight) {
    GradientTables T;
    T.logt = second ? logt1 : logt0;
    const nrb_objective *last = second ? last1 : last0;
    T.nmi = last->nmi;
    T.scale = weight / (last->entropy[2] * last->entropy[3]);
    T.nmi_f = (float)T.nmi;
    T.scale_f = (float)T.scale;
    return T;
}

// FP32 copy of the log table in shared memory for the FP32 window (visible after the next
// stage_item barrier)
__device__ __forceinline__ void stage_log_table(const WalkParams& P, const double *logt, float *logf) {
    const int total = P.rb * P.fb + P.rb + P.fb;
    for (int i = threadIdx.x; i < total; i += blockDim.x) logf[i] = (float)logt[i];
}

// One item of the fused gradient: stage the item's control points, walk its columns and write
// every voxel's NMI gradient (zero where masked or NaN). Called by every thread of the block.
template <bool kF32, bool kDiag>
__device__ __forceinline__ void gradient_item(const WalkParams& P, const WalkSmem& S, const float *logf,
                                              const GradientTables& T, int item, const float *__restrict__ ref,
                                              const float *__restrict__ flo, const int32_t *__restrict__ mask,
                                              const float *__restrict__ cpp, float *__restrict__ vgrad) {
    const int nv = P.nx * P.ny * P.nz;
    Item I;
    stage_item(P, cpp, item, S.cp, S.zb, S.zk, S.zid, I);
    Column C;
    column_init(P, I, S.cp, C);
    const int nzi = I.z1 - I.z0;
    const int zstride = P.nx * P.ny;
    int idx = (I.z0 * P.ny + C.y) * P.nx + C.x;
    for (int zi = 0; zi < nzi; ++zi, idx += zstride) {
        float pos[3];
        column_position(P, I, C, S.zb, S.zk, S.zid, zi, pos);
        if (!C.inside) continue;
        float out[3] = { 0.f, 0.f, 0.f };
        if (mask == nullptr || __ldg(&mask[idx]) > -1) {
            float w, g[3];
            sample_floating<true, kDiag ? 1 : 0>(flo, P.ftex, P.fnx, P.fny, P.fnz, P.fsy, P.fsz, P.fmargin, P.flo_ijk,
                                                 P.flo_diag, P.pad, pos[0], pos[1], pos[2], w, g);
            const float rv = __ldg(&ref[idx]);
            if (rv == rv && w == w) {
                if (kF32) {
                    const float s = nmi_window_f(rv, w, logf, P.rb, P.fb, T.nmi_f);
#pragma unroll
                    for (int d = 0; d < 3; ++d) out[d] = T.scale_f * (g[d] * s);
                } else {
                    const double s = nmi_window(rv, w, T.logt, P.rb, P.fb, T.nmi);
#pragma unroll
                    for (int d = 0; d < 3; ++d) out[d] = (float)(T.scale * ((double)g[d] * s));
                }
            }
        }
        vgrad[idx] = out[0];
        vgrad[nv + idx] = out[1];
        vgrad[2 * nv + idx] = out[2];
    }
}

template <bool kF32, bool kDiag>
__global__ void __launch_bounds__(32 * TY_GRADIENT, kF32 ? 6 : 4)
k_gradient(WalkParams P, const float *__restrict__ ref, const float *__restrict__ flo,
           const int32_t *__restrict__ mask, const float *__restrict__ cpp,
           const double *logt0, const nrb_objective *last0, const double *logt1, const nrb_objective *last1,
           const OptState *__restrict__ sel, double weight, float *__restrict__ vgrad) {
    extern __shared__ float4 sm4[];
    const WalkSmem S = walk_smem(P, sm4);
    const GradientTables T = gradient_tables(logt0, last0, logt1, last1, sel && sel->best_buf == 1, weight);
    float *logf = reinterpret_cast<float *>(S.tail);
    if (kF32) stage_log_table(P, T.logt, logf);
    for (int item = blockIdx.x; item < P.nitems; item += gridDim.x)
        gradient_item<kF32, kDiag>(P, S, logf, T, item, ref, flo, mask, cpp, vgrad);
}

// standalone deformation field (Compute::GetDeformationField) with the same arithmetic
__global__ void __launch_bounds__(32 * TY_DEFORMATION)
k_deformation(WalkParams P, const int32_t *__restrict__ mask, const float *__restrict__ cpp,
              float *__restrict__ def) {
    extern __shared__ float4 sm4[];
    const WalkSmem S = walk_smem(P, sm4);
    const int nv = P.nx * P.ny * P.nz;
    for (int item = blockIdx.x; item < P.nitems; item += gridDim.x) {
        Item I;
        stage_item(P, cpp, item, S.cp, S.zb, S.zk, S.zid, I);
        Column C;
        column_init(P, I, S.cp, C);
        const int nzi = I.z1 - I.z0;
        for (int zi = 0; zi < nzi; ++zi) {
            float pos[3];
            column_position(P, I, C, S.zb, S.zk, S.zid, zi, pos);
            if (!C.inside) continue;
            const int idx = ((I.z0 + zi) * P.ny + C.y) * P.nx + C.x;
            if (mask != nullptr && __ldg(&mask[idx]) <= -1) pos[0] = pos[1] = pos[2] = 0.f;
            def[idx] = pos[0];
            def[nv + idx] = pos[1];
            def[2 * nv + idx] = pos[2];
        }
    }
}


// ---------------------------------------------------------------------------------------------
// histogram -> smoothed probabilities, FP64 entropies, log table (one cluster, tables in smem)
// ---------------------------------------------------------------------------------------------
// one 3-tap smoothing output in the reference's accumulation order (value = 0; value +=
// left*k0; value += centre*k1; value += right*k0, in-range taps only), no contraction
__device__ __forceinline__ double smooth3(bool has_l, double l, double m, bool has_r, double r, double k0, double k1) {
    double v = 0.0;
    if (has_l) v = __dadd_rn(v, __dmul_rn(l, k0));
    v = __dadd_rn(v, __dmul_rn(m, k1));
    if (has_r) v = __dadd_rn(v, __dmul_rn(r, k0));
    return v;
}

// fixed-shape block sum of three doubles over NW warps
template <int NW>
__device__ __forceinline__ void block_sum3w(double& a, double& b, double& c, double *red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
    }
    __syncthreads();  // red is free
    if (lane == 0) {
        red[3 * wid] = a;
        red[3 * wid + 1] = b;
        red[3 * wid + 2] = c;
    }
    __syncthreads();
    if (wid == 0) {
        a = lane < NW ? red[3 * lane] : 0.0;
        b = lane < NW ? red[3 * lane + 1] : 0.0;
        c = lane < NW ? red[3 * lane + 2] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
            c += __shfl_down_sync(0xffffffffu, c, o);
        }
        if (lane == 0) {
            red[0] = a;
            red[1] = b;
            red[2] = c;
        }
    }
    __syncthreads();
    a = red[0];
    b = red[1];
    c = red[2];
}

// _reg_nmi.cpp:249-346 with the histogram as integer counts: 3-tap [1/6, float(2/3), 1/6]
// smoothing along the reference axis then the floating axis (each entry bit-identical to the
// reference's), normalisation by the total, marginals, entropies and the log table. The
// bending-energy partials of the same evaluation are summed here too.
//
// One cluster of FIN_CLUSTER blocks: block c owns the floating-bin rows [c*rpc, (c+1)*rpc) of
// the joint table (rows are reference-bin contiguous). It smooths its rows (reading one halo row
// of counts on each side) and the blocks exchange partial sums (mass, reference marginal,
// entropies) through distributed shared memory, always combined in block order. Shared memory
// per block: T = own rows, U = own rows + 2 halo rows (later the partial reference marginal).
constexpr int FIN_CLUSTER = 8, FIN_CTA_THREADS = 256, FIN_WARPS = FIN_CTA_THREADS / 32;

// What the finalize does besides the tables: FIN_PLAIN a standalone evaluation (table set 0, no
// optimiser); FIN_LINE a line-search step of a level graph (line_step, the line search's WHILE
// condition); FIN_BATCH_INIT / FIN_BATCH_LINE the same two inside a batched level, where the
// pair's phase moves on instead of a condition being set (INIT: the starting point's values
// become the best ones; LINE: line_step, then the end of the line search when it stops).
enum FinMode : int { FIN_PLAIN = 0, FIN_LINE = 1, FIN_BATCH_INIT = 2, FIN_BATCH_LINE = 3 };

struct FinArgs {
    int rb, fb;
    uint32_t *hist;
    double *pro0, *logt0;
    nrb_objective *last0;
    double *pro1, *logt1;
    nrb_objective *last1;
    const double *be_partials;
    int n_be;
    double be_norm, sim_weight, be_weight;
    nrb_objective *obj;
    OptState *ctl;
    float *acc_best;
    const float *acc_grad;
    long long acc_n;
};

template <int kMode>
__device__ __forceinline__ void finalize_cluster(cg::cluster_group& cluster, const FinArgs& A,
                                                 cudaGraphConditionalHandle line) {
    const int rb = A.rb, fb = A.fb;
    uint32_t *__restrict__ hist = A.hist;
    const double *__restrict__ be_partials = A.be_partials;
    const int n_be = A.n_be;
    const double be_norm = A.be_norm, sim_weight = A.sim_weight, be_weight = A.be_weight;
    nrb_objective *__restrict__ obj = A.obj;
    OptState *__restrict__ ctl = A.ctl;
    nrb_objective *last0 = A.last0, *last1 = A.last1;
    extern __shared__ double sm[];
    __shared__ double red[3 * 32];
    __shared__ double part[4];  // this block's partial mass, H_ref, H_war, H_joint
    __shared__ OptState sctl;   // this block's copy of the optimiser state
    __shared__ double s_mgl[2];
    const int tid = threadIdx.x, c = (int)cluster.block_rank();
    // threads beyond FIN_CTA_THREADS (a caller with larger blocks) take part in the barriers only,
    // so the work and its summation order are those of FIN_CTA_THREADS-thread blocks
    const bool act = tid < FIN_CTA_THREADS;
    // everything the end of the kernel needs from global memory is read now, beside the counts:
    // the optimiser state, the gradient lengths of both table sets, the bending-energy partials
    // (counts and partials through L2: other blocks of the same launch may have written them)
    if (tid == 0) {
        if (ctl) sctl = *ctl;
        s_mgl[0] = last0->max_grad_len;
        s_mgl[1] = last1->max_grad_len;
    }
    double be = 0.0;
    if (act)
        for (int i = tid; i < n_be; i += FIN_CTA_THREADS) be += __ldcg(&be_partials[i]);
    // the state and the partials come from earlier launches (the bending-energy pass is a full
    // dependency); the counts from the objective pass this launch may have started beside
    pdl_wait();
    const int nj = rb * fb;
    const int rpc = (fb + FIN_CLUSTER - 1) / FIN_CLUSTER;
    const int f0 = min(fb, c * rpc), f1 = min(fb, f0 + rpc), nrow = f1 - f0;
    double *T = sm;               // rpc rows
    double *U = sm + rpc * rb;    // rpc + 2 rows: U row k = floating bin f0 - 1 + k
    const double k0 = parzen(-1.0), k1 = parzen(0.0);
    // smoothing along the reference axis straight from the integer counts, own rows + halo
    const int ua = max(0, f0 - 1), ub = min(fb, f1 + 1);
    if (act)
        for (int i = tid; i < (ub - ua) * rb; i += FIN_CTA_THREADS) {
            const int f = ua + i / rb, r = i % rb;
            const uint32_t *row = hist + (size_t)f * rb;
            const double m = (double)__ldcg(&row[r]);
            const double l = r > 0 ? (double)__ldcg(&row[r - 1]) : 0.0;
            const double rr = r + 1 < rb ? (double)__ldcg(&row[r + 1]) : 0.0;
            U[(f - f0 + 1) * rb + r] = smooth3(r > 0, l, m, r + 1 < rb, rr, k0, k1);
        }
    __syncthreads();
    // output table set: the one not holding the best position (a level's starting point and a
    // standalone evaluation write the first set)
    const bool second = (kMode == FIN_LINE || kMode == FIN_BATCH_LINE) && sctl.best_buf == 0;
    double *__restrict__ pro = second ? A.pro1 : A.pro0;
    double *__restrict__ logt = second ? A.logt1 : A.logt0;
    nrb_objective *__restrict__ last = second ? last1 : last0;
    // smoothing along the floating axis of the own rows
    double mass = 0.0, z2 = 0.0;
    if (act)
        for (int i = tid; i < nrow * rb; i += FIN_CTA_THREADS) {
            const int f = f0 + i / rb;
            const double *u = U + (i / rb + 1) * rb + i % rb;
            const double v = smooth3(f > 0, f > 0 ? u[-rb] : 0.0, u[0], f + 1 < fb, f + 1 < fb ? u[rb] : 0.0, k0, k1);
            T[i] = v;
            mass += v;
        }
    // the bending-energy sum: the same partition and tree in every block, so the same value
    block_sum3w<FIN_WARPS>(mass, be, z2, red);
    if (tid == 0) part[0] = mass;
    cluster.sync();  // every block has read its halo counts; partial masses visible
    if (act)
        for (int i = tid; i < nrow * rb; i += FIN_CTA_THREADS) hist[(size_t)f0 * rb + i] = 0u;  // next evaluation
    double total = 0.0;
    {
        double pq[FIN_CLUSTER];
#pragma unroll
        for (int q = 0; q < FIN_CLUSTER; ++q) pq[q] = cluster.map_shared_rank(part, q)[0];  // in flight together
#pragma unroll
        for (int q = 0; q < FIN_CLUSTER; ++q) total += pq[q];
    }
    // normalised own rows, their logs and the joint entropy
    double hj = 0.0;
    if (act)
        for (int i = tid; i < nrow * rb; i += FIN_CTA_THREADS) {
            const double p = T[i] / total;
            T[i] = p;
            double l = 0.0;
            if (p > 0) {
                l = log(p);
                hj -= p * l;
            }
            pro[(size_t)f0 * rb + i] = p;
            logt[(size_t)f0 * rb + i] = l;
        }
    __syncthreads();
    // partial reference marginal over the own rows (U is free now), in floating-bin order
    double *R = U;
    if (act)
        for (int r = tid; r < rb; r += FIN_CTA_THREADS) {
            double sum = 0.0;
            for (int k = 0; k < nrow; ++k) sum += T[k * rb + r];
            R[r] = sum;
        }
    // floating marginal of the own rows: eight lanes per row, each summing a strided share of the
    // reference bins, combined by shuffles in a fixed order
    double hw = 0.0;
    if (act) {  // whole warps: the shuffles below stay within active warps
        const int sub = tid & 7;
        // the trip count is the same for every thread, so all lanes reach the shuffles
        for (int k0 = 0; k0 < rpc; k0 += FIN_CTA_THREADS / 8) {
            const int k = k0 + (tid >> 3);
            double sum = 0.0;
            if (k < nrow)
                for (int r = sub; r < rb; r += 8) sum += T[k * rb + r];
            sum += __shfl_xor_sync(0xffffffffu, sum, 1);
            sum += __shfl_xor_sync(0xffffffffu, sum, 2);
            sum += __shfl_xor_sync(0xffffffffu, sum, 4);
            if (sub == 0 && k < nrow) {
                double l = 0.0;
                if (sum > 0) {
                    l = log(sum);
                    hw -= sum * l;
                }
                pro[nj + rb + f0 + k] = sum;
                logt[nj + rb + f0 + k] = l;
            }
        }
    }
    cluster.sync();  // partial reference marginals of every block visible
    // reference marginal: the blocks' partial sums added in block order (a fixed order, so the
    // result repeats bit for bit; it differs from a sequential sum only in the last bits)
    double hr = 0.0;
    for (int r = c + FIN_CLUSTER * tid; act && r < rb; r += FIN_CLUSTER * FIN_CTA_THREADS) {
        double rq[FIN_CLUSTER];
#pragma unroll
        for (int q = 0; q < FIN_CLUSTER; ++q) rq[q] = cluster.map_shared_rank(R, q)[r];
        double sum = 0.0;
#pragma unroll
        for (int q = 0; q < FIN_CLUSTER; ++q) sum += rq[q];
        double l = 0.0;
        if (sum > 0) {
            l = log(sum);
            hr -= sum * l;
        }
        pro[nj + r] = sum;
        logt[nj + r] = l;
    }
    block_sum3w<FIN_WARPS>(hr, hw, hj, red);
    if (tid == 0) {
        part[1] = hr;
        part[2] = hw;
        part[3] = hj;
    }
    cluster.sync();
    if (tid == 0) {
        double hq[FIN_CLUSTER][3];
#pragma unroll
        for (int q = 0; q < FIN_CLUSTER; ++q) {
            const double *pq = cluster.map_shared_rank(part, q);
            hq[q][0] = pq[1];
            hq[q][1] = pq[2];
            hq[q][2] = pq[3];
        }
        double h[3] = { 0.0, 0.0, 0.0 };
#pragma unroll
        for (int q = 0; q < FIN_CLUSTER; ++q) {
            h[0] += hq[q][0];
            h[1] += hq[q][1];
            h[2] += hq[q][2];
        }
        nrb_objective o;
        // with a zero similarity weight the reference never evaluates the measure
        // (_reg_f3d.cpp:450-454): its weighted term is 0, not 0 * NaN
        o.nmi = sim_weight > 0 ? (h[0] + h[1]) / h[2] : 0.0;
        o.entropy[0] = h[0];
        o.entropy[1] = h[1];
        o.entropy[2] = h[2];
        o.entropy[3] = total;
        o.be = n_be > 0 ? be / be_norm : 0.0;
        o.objective = (sim_weight > 0 ? sim_weight * o.nmi : 0.0) - (be_weight > 0 ? be_weight * o.be : 0.0);
        o.max_grad_len = s_mgl[second ? 1 : 0];
        // every block takes the same step on its own copy of the state; block 0 publishes it
        bool more = false;
        if (kMode == FIN_LINE || kMode == FIN_BATCH_LINE) more = line_step(&sctl, o.nmi, o.be, sim_weight, be_weight);
        if (kMode == FIN_BATCH_INIT) {
            // ConjugateGradient::Initialise: the starting point is the best one so far
            // (reg_f3d::GetObjectiveFunctionValue's weighted terms, as line_step forms them)
            const double wm = sim_weight > 0 ? sim_weight * o.nmi : 0.0;
            const double wb = be_weight > 0 ? be_weight * o.be : 0.0;
            sctl.n_obj += 1;
            sctl.best_w_measure = wm;
            sctl.best_w_be = wb;
            sctl.best_nmi = o.nmi;
            sctl.best_be = o.be;
            sctl.best_obj = __dsub_rn(wm, wb);
            sctl.accepted = 0;
            sctl.phase = outer_continues(sctl) ? PH_GRAD : PH_DONE;
        }
        if (kMode == FIN_BATCH_LINE && !more) sctl.phase = line_end(&sctl) ? PH_GRAD : PH_DONE;
        if (c == 0) {
            *last = o;
            if (obj) *obj = o;
            if (kMode != FIN_PLAIN) *ctl = sctl;
            if (kMode == FIN_LINE) cudaGraphSetConditional(line, more ? 1u : 0u);
        }
    }
    // this block has read the others' shared memory: they may exit once every block arrived
    auto token = cluster.barrier_arrive();
    __syncthreads();  // the decision in sctl
    // the store of an accepted trial position (k_accept's operations) in the same launch
    if ((kMode == FIN_LINE || kMode == FIN_BATCH_LINE) && A.acc_n > 0 && sctl.accepted && act) {
        const float scale = -sctl.step_len;
        for (long long i = (long long)c * FIN_CTA_THREADS + tid; i < A.acc_n;
             i += (long long)FIN_CLUSTER * FIN_CTA_THREADS)
            A.acc_best[i] = __fadd_rn(A.acc_best[i], __fmul_rn(scale, A.acc_grad[i]));
    }
    cluster.barrier_wait(std::move(token));
}

__global__ void __cluster_dims__(FIN_CLUSTER, 1, 1) __launch_bounds__(FIN_CTA_THREADS)
k_nmi_finalize(FinArgs A, cudaGraphConditionalHandle line) {
    pdl_launch_dependents();  // the store of an accepted position (large grids) may queue behind it
    cg::cluster_group cluster = cg::this_cluster();
    if (A.ctl) finalize_cluster<FIN_LINE>(cluster, A, line);
    else finalize_cluster<FIN_PLAIN>(cluster, A, line);
}

// ---------------------------------------------------------------------------------------------
// standalone resampling / histogram / voxel gradient (materialised intermediates)
// ---------------------------------------------------------------------------------------------
template <bool kGrad>
__global__ void k_resample(long long nv, int fnx, int fny, int fnz, Mat34 M, int diag, float pad,
                           const float *__restrict__ flo, const float *__restrict__ def,
                           const int32_t *__restrict__ mask, float *__restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
         i += (long long)gridDim.x * blockDim.x) {
        const bool active = mask == nullptr || mask[i] > -1;
        if (!kGrad && !active) continue;
        float w = 0.f, g[3] = { 0.f, 0.f, 0.f };
        if (active)
            sample_floating<kGrad>(flo, 0ull, fnx, fny, fnz, fnx, fnx * fny, 0, M, diag, pad, def[i], def[nv + i],
                                   def[2 * nv + i], w, g);
        if (kGrad) {
            out[i] = g[0];
            out[nv + i] = g[1];
            out[2 * nv + i] = g[2];
        } else {
            out[i] = w;
        }
    }
}

// Weights of the resampling kernels of order 0 (nearest), 1 (linear) and 3 (cubic spline), as
// interpNearestNeighKernel / interpLinearKernel / interpCubicSplineKernel compute them
// (reg-lib/cpu/_reg_resampling.cpp:60-97): float, every product and sum rounded on its own.
template <int kOrder>
__device__ __forceinline__ void order_weights(float rel, float w[4]) {
    if (rel < 0.f) rel = 0.f;  // the kernels' rounding guard
    if (kOrder == 0) {
        w[0] = rel >= 0.5f ? 0.f : 1.f;
        w[1] = rel >= 0.5f ? 1.f : 0.f;
    } else if (kOrder == 1) {
        w[1] = rel;
        w[0] = __fsub_rn(1.f, rel);
    } else {
        const float sq = __fmul_rn(rel, rel);
        w[0] = __fmul_rn(__fmul_rn(rel, __fsub_rn(__fmul_rn(__fsub_rn(2.f, rel), rel), 1.f)), 0.5f);
        w[1] = __fmul_rn(__fadd_rn(__fmul_rn(sq, __fsub_rn(__fmul_rn(3.f, rel), 5.f)), 2.f), 0.5f);
        w[2] = __fmul_rn(__fmul_rn(rel, __fadd_rn(__fmul_rn(__fsub_rn(4.f, __fmul_rn(3.f, rel)), rel), 1.f)), 0.5f);
        w[3] = __fmul_rn(__fmul_rn(__fsub_rn(rel, 1.f), sq), 0.5f);
    }
}

// ResampleImage3D with the kernel of order kOrder (reg-lib/cpu/_reg_resampling.cpp:316-464) at
// world position (x, y, z), with the reference's operations: mm -> voxel as Mat44Mul (products of
// two floats are exact in double), a window of 2 (orders 0, 1) or 4 (order 3, starting one voxel
// before floor) taps per axis, sums in float along x, then y, then z, and padding * weight for
// every out-of-volume tap when the window leaves the volume. Bit-identical to the reference.
template <int kOrder>
__device__ __forceinline__ float sample_order(const float *__restrict__ flo, int fnx, int fny, int fnz,
                                              const Mat34& M, float pad, float x, float y, float z) {
    constexpr int kTaps = kOrder == 3 ? 4 : 2, kOffset = kOrder == 3 ? 1 : 0;
    float fx, fy, fz;
    to_floating_voxel<0>(M, 0, x, y, z, fx, fy, fz);
    const float fp[3] = { fx, fy, fz };
    float w[3][4];
    int first[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float fl = floorf(fp[d]);
        order_weights<kOrder>(__fsub_rn(fp[d], fl), w[d]);
        first[d] = (int)fl - kOffset;
    }
    // tap indices in unsigned arithmetic: a window far outside (a saturated floor) wraps to
    // indices that fail the range tests instead of overflowing
    const unsigned ux = (unsigned)first[0], uy = (unsigned)first[1], uz = (unsigned)first[2];
    const bool inside = first[0] > -1 && ux + (kTaps - 1) < (unsigned)fnx && first[1] > -1 &&
                        uy + (kTaps - 1) < (unsigned)fny && first[2] > -1 && uz + (kTaps - 1) < (unsigned)fnz;
    float intensity = 0.f;
#pragma unroll
    for (int c = 0; c < kTaps; ++c) {
        const unsigned Z = uz + c;
        float yv = 0.f;
#pragma unroll
        for (int b = 0; b < kTaps; ++b) {
            const unsigned Y = uy + b;
            float xv = 0.f;
#pragma unroll
            for (int a = 0; a < kTaps; ++a) {
                const unsigned X = ux + a;
                const bool in = inside || (X < (unsigned)fnx && Y < (unsigned)fny && Z < (unsigned)fnz);
                const float v = in ? __ldg(flo + ((long long)Z * fny + Y) * fnx + X) : pad;
                xv = __fadd_rn(xv, __fmul_rn(v, w[0][a]));
            }
            yv = __fadd_rn(yv, __fmul_rn(xv, w[1][b]));
        }
        intensity = __fadd_rn(intensity, __fmul_rn(yv, w[2][c]));
    }
    return intensity;
}

// sample_order at the positions of a deformation field, one voxel per thread; masked voxels keep
// their value
template <int kOrder>
__global__ void k_resample_order(long long nv, int fnx, int fny, int fnz, Mat34 M, float pad,
                                 const float *__restrict__ flo, const float *__restrict__ def,
                                 const int32_t *__restrict__ mask, float *__restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
         i += (long long)gridDim.x * blockDim.x) {
        if (mask != nullptr && mask[i] <= -1) continue;
        out[i] = sample_order<kOrder>(flo, fnx, fny, fnz, M, pad, def[i], def[nv + i], def[2 * nv + i]);
    }
}

// The final warp in one pass: k_deformation's positions (the same column walk, so the same
// floats) consumed at once by sample_order; the deformation field never reaches memory.
template <int kOrder>
__global__ void __launch_bounds__(32 * TY_DEFORMATION)
k_warp_order(WalkParams P, const float *__restrict__ cpp, const float *__restrict__ flo, float *__restrict__ warped) {
    extern __shared__ float4 sm4[];
    const WalkSmem S = walk_smem(P, sm4);
    for (int item = blockIdx.x; item < P.nitems; item += gridDim.x) {
        Item I;
        stage_item(P, cpp, item, S.cp, S.zb, S.zk, S.zid, I);
        Column C;
        column_init(P, I, S.cp, C);
        const int nzi = I.z1 - I.z0;
        for (int zi = 0; zi < nzi; ++zi) {
            float pos[3];
            column_position(P, I, C, S.zb, S.zk, S.zid, zi, pos);
            if (!C.inside) continue;
            const int idx = ((I.z0 + zi) * P.ny + C.y) * P.nx + C.x;
            warped[idx] = sample_order<kOrder>(flo, P.fnx, P.fny, P.fnz, P.flo_ijk, P.pad, pos[0], pos[1], pos[2]);
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
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
         i += (long long)gridDim.x * blockDim.x) {
        if (mask != nullptr && mask[i] <= -1) continue;
        const float r = ref[i], w = war[i];
        if (r == r && w == w && 0.f <= r && r < (float)rb && 0.f <= w && w < (float)fb)
            atomicAdd(&hs[(int)r + (int)w * rb], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nbins; i += blockDim.x) {
        const uint32_t v = hs[i];
        if (v) atomicAdd(&ghist[i], v);
    }
}

// kF32: the Parzen window in FP32 on an FP32 copy of the log table in shared memory, as the fused
// gradient runs it (the normalisation constant formed in FP64); otherwise the FP64 window on the
// global table (tables too large for shared memory).
template <bool kF32>
__global__ void k_nmi_voxel_gradient(long long nv, int rb, int fb, const float *__restrict__ ref,
                                     const float *__restrict__ war, const float *__restrict__ wgrad,
                                     const int32_t *__restrict__ mask, const double *__restrict__ logt,
                                     const nrb_objective *__restrict__ last, double weight,
                                     float *__restrict__ vgrad) {
    extern __shared__ float logf_sm[];
    const double nmi = last->nmi;
    const double scale = weight / (last->entropy[2] * last->entropy[3]);
    const float nmi_f = (float)nmi, scale_f = (float)scale;
    if (kF32) {
        const int total = rb * fb + rb + fb;
        for (int i = threadIdx.x; i < total; i += blockDim.x) logf_sm[i] = (float)logt[i];
        __syncthreads();
    }
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
         i += (long long)gridDim.x * blockDim.x) {
        if (mask != nullptr && mask[i] <= -1) continue;
        const float r = ref[i], w = war[i];
        if (!(r == r && w == w)) continue;
        if (kF32) {
            const float s = nmi_window_f(r, w, logf_sm, rb, fb, nmi_f);
            for (int d = 0; d < 3; ++d) {
                const float g = wgrad[d * nv + i];
                if (g == g) vgrad[d * nv + i] += scale_f * (g * s);
            }
        } else {
            const double s = nmi_window(r, w, logt, rb, fb, nmi);
            for (int d = 0; d < 3; ++d) {
                const float g = wgrad[d * nv + i];
                if (g == g) vgrad[d * nv + i] += (float)(scale * ((double)g * s));
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// batched levels: one launch per stage over every pair that needs it
// ---------------------------------------------------------------------------------------------
// The objective of every pair in INIT (at best) or LINE (at best - cur_len * grad): each block
// walks its share of the pairs' items with the pair's own walk and histogram, exactly the
// plain k_objective's work per item.
template <bool kXs, bool kDiag>
__global__ void __launch_bounds__(32 * TY_OBJECTIVE, 2)
k_b_objective(const __grid_constant__ BatchObjTable T, const OptState *__restrict__ states, int npairs) {
    extern __shared__ float4 sm4[];
    __shared__ BatchList L;
    __shared__ BatchSegments G;
    batch_list_build(states, npairs, (1u << PH_INIT) | (1u << PH_LINE),
                     [&](int q, int& u, int& w) {
                         u = T.e[q].P.nitems;
                         w = T.e[q].P.zchunk + 6;
                     }, L);
    batch_segments(L, G);
    for (int sg = 0; sg < G.n; ++sg) {
        const int p = G.pair[sg];
        WalkSmem S;
        uint32_t *h;
        float *X;
        objective_smem(T.e[p].P, sm4, S, h, X);
        const int nbins = T.e[p].P.rb * T.e[p].P.fb;
        __syncthreads();  // the previous pair's flush has read the shared histogram
        zero_hist(h, nbins);  // ordered before the counts by stage_item's first barrier
        for (int j = G.j0[sg]; j < G.j1[sg]; ++j) {
            const int q = G.pair[sg];
            const bool line = states[q].phase == PH_LINE;
            objective_item<kXs, kDiag>(T.e[q].P, S, h, X, j, T.e[q].ref, T.e[q].flo, nullptr, T.e[q].best,
                                       line ? T.e[q].grad : nullptr, line ? -states[q].cur_len : 0.f);
        }
        flush_hist(h, nbins, T.e[G.pair[sg]].hist);
    }
}

// The fused voxel gradient of every pair in GRAD, at best, with the NMI tables of its best
// position (the plain k_gradient's work per item).
template <bool kF32, bool kDiag>
__global__ void __launch_bounds__(32 * TY_GRADIENT, kF32 ? 6 : 4)
k_b_gradient(const __grid_constant__ BatchGradTable T, const OptState *__restrict__ states, int npairs) {
    extern __shared__ float4 sm4[];
    __shared__ BatchList L;
    __shared__ BatchSegments G;
    batch_list_build(states, npairs, 1u << PH_GRAD,
                     [&](int q, int& u, int& w) {
                         u = T.e[q].P.nitems;
                         w = T.e[q].P.zchunk + 4;
                     }, L);
    batch_segments(L, G);
    for (int sg = 0; sg < G.n; ++sg) {
        const int p = G.pair[sg];
        const BatchGradEntry& E = T.e[p];
        const WalkSmem S = walk_smem(E.P, sm4);
        const GradientTables N = gradient_tables(E.logt0, E.last0, E.logt1, E.last1, states[p].best_buf == 1, 1.0);
        float *logf = reinterpret_cast<float *>(S.tail);
        __syncthreads();  // the previous pair's walk is done with the shared tables
        if (kF32) stage_log_table(E.P, N.logt, logf);  // visible after stage_item's first barrier
        for (int j = G.j0[sg]; j < G.j1[sg]; ++j)
            gradient_item<kF32, kDiag>(E.P, S, logf, N, j, E.ref, E.flo, nullptr, E.best, E.vgrad);
    }
}

// One finalize cluster per pair (cluster q = pair q): the pairs in INIT or LINE finish their
// evaluation (tables, NMI, bending energy, line-search step, accepted step stored, phase moved
// on); the last cluster sets whether the gradient stage runs this iteration (enough pairs wait
// for it, or no pair has a line-search step left) and whether the level goes on.
__global__ void __cluster_dims__(FIN_CLUSTER, 1, 1) __launch_bounds__(FIN_CTA_THREADS)
k_b_finalize(const BatchPair *__restrict__ pairs, OptState *__restrict__ states, int npairs,
             BatchCtl *__restrict__ bctl, int in_graph, cudaGraphConditionalHandle grad_if,
             cudaGraphConditionalHandle outer) {
    pdl_wait();  // the counts come from the objective pass
    cg::cluster_group cluster = cg::this_cluster();
    const int p = blockIdx.x / FIN_CLUSTER;
    const int phase = states[p].phase;
    if (phase == PH_INIT || phase == PH_LINE) {
        const BatchPair& B = pairs[p];
        FinArgs A;
        A.rb = B.rb;
        A.fb = B.fb;
        A.hist = B.hist;
        A.pro0 = B.pro0;
        A.logt0 = B.logt0;
        A.last0 = B.last0;
        A.pro1 = B.pro1;
        A.logt1 = B.logt1;
        A.last1 = B.last1;
        A.be_partials = B.be_partials;
        A.n_be = B.be_w > 0 ? B.n_be : 0;
        A.be_norm = B.be_norm;
        A.sim_weight = B.sim_w;
        A.be_weight = B.be_w;
        A.obj = B.obj;
        A.ctl = &states[p];
        A.acc_best = B.best;
        A.acc_grad = B.grad;
        A.acc_n = 3 * B.nnode;
        if (phase == PH_INIT) finalize_cluster<FIN_BATCH_INIT>(cluster, A, 0);
        else finalize_cluster<FIN_BATCH_LINE>(cluster, A, 0);
    }
    if (cluster.block_rank() != 0) return;
    if (!batch_last_cluster(&bctl->ticket_fin, gridDim.x / FIN_CLUSTER)) return;
    int nline, ngrad;
    batch_counts(states, npairs, nline, ngrad);
    if (threadIdx.x == 0) {
        const bool run_grad = ngrad > 0 && (100 * ngrad >= bctl->grad_percent * (nline + ngrad) || nline == 0);
        if (in_graph) {
            cudaGraphSetConditional(grad_if, run_grad ? 1u : 0u);
            cudaGraphSetConditional(outer, nline + ngrad > 0 ? 1u : 0u);
        }
        bctl->run_grad = run_grad;
        bctl->go_on = nline + ngrad > 0;
        bctl->iterations += 1;
        bctl->grad_stages += run_grad ? 1 : 0;
    }
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
static WalkParams make_params(const WalkPlan& W, const nrb_geometry *g, float pad, int rb, int fb) {
    WalkParams P{};
    P.nx = g->ref_dim[0];
    P.ny = g->ref_dim[1];
    P.nz = g->ref_dim[2];
    P.cx = g->cpp_dim[0];
    P.cy = g->cpp_dim[1];
    P.cz = g->cpp_dim[2];
    P.gsx = g->cpp_pixdim[0] / g->ref_pixdim[0];
    P.gsy = g->cpp_pixdim[1] / g->ref_pixdim[1];
    P.gsz = g->cpp_pixdim[2] / g->ref_pixdim[2];
    P.ty = W.ty;
    P.tiles_x = W.tiles_x;
    P.tiles_y = W.tiles_y;
    P.zchunk = W.zchunk;
    P.nitems = W.nitems;
    P.sa = W.sa;
    P.sb = W.sb;
    P.sc = W.sc;
    P.fnx = g->flo_dim[0];
    P.fny = g->flo_dim[1];
    P.fnz = g->flo_dim[2];
    P.fsy = P.fnx;
    P.fsz = P.fnx * P.fny;
    P.fmargin = 0;
    P.flo_ijk = to_mat34(g->flo_ijk);
    P.pad = pad;
    P.rb = rb;
    P.fb = fb;
    P.cnv = P.cx * P.cy * P.cz;
    const float *m = g->flo_ijk;
    P.flo_diag = m[1] == 0.f && m[2] == 0.f && m[4] == 0.f && m[6] == 0.f && m[8] == 0.f && m[9] == 0.f;
    P.log_in_smem = 0;
    P.xs = 0;
    P.ftex = 0;
    // identity split when the grid's voxel -> mm matrix has no off-diagonal terms
    const float *c = g->cpp_xyz;
    const bool cdiag = c[1] == 0.f && c[2] == 0.f && c[4] == 0.f && c[6] == 0.f && c[8] == 0.f && c[9] == 0.f;
    for (int d = 0; d < 3; ++d) {
        P.io[d] = cdiag ? c[4 * d + 3] : 0.f;
        P.is[d] = cdiag ? c[5 * d] : 0.f;
    }
    return P;
}

// a floating image laid out by pad_volume with `margin` voxels on every side, passed as the
// pointer to its voxel (0, 0, 0)
static void set_floating_margin(WalkParams& P, int margin) {
    P.fmargin = margin;
    P.fsy = P.fnx + 2 * margin;
    P.fsz = P.fsy * (P.fny + 2 * margin);
}

template <typename K>
static nrb_status persistent_grid(K kernel, int threads, size_t smem, int nitems, int& grid, int resident = 0) {
    NRB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    if (resident <= 0) {
        int per_sm = 0;
        NRB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
        resident = per_sm * sm_count();
    }
    if (resident < 1) return fail(NRB_ERR_UNSUPPORTED, "voxel walk does not fit in shared memory");
    // every block gets the same number of items: as many rounds as the resident blocks need,
    // then the smallest grid that covers the items in that many rounds
    const int rounds = (nitems + resident - 1) / resident;
    grid = (nitems + rounds - 1) / rounds;
    return NRB_OK;
}

template <typename K>
static long long blocks_resident(K kernel, int threads, size_t smem) {
    int per_sm = 0;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return (long long)per_sm * sm_count();
}

long long objective_slots(size_t smem) { return blocks_resident(k_objective<true, true, true>, 32 * TY_OBJECTIVE, smem); }
long long gradient_slots(size_t smem) { return blocks_resident(k_gradient<true, true>, 32 * TY_GRADIENT, smem); }
long long deformation_slots(size_t smem) { return blocks_resident(k_deformation, 32 * TY_DEFORMATION, smem); }

nrb_status launch_fused_objective(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g,
                                  const float *ref, const float *flo, const int32_t *mask,
                                  const float *cpp, float padding, cudaStream_t st,
                                  const float *grad, const OptState *step, int flo_margin) {
    WalkParams P = make_params(ws->walk_obj, g, padding, nmi->rb, nmi->fb);
    set_floating_margin(P, flo_margin);
    P.ftex = flo_margin >= 2 ? ws->flo_tex : 0ull;
    const size_t base_smem = walk_smem_bytes(ws->walk_obj) + (size_t)((nmi->rb * nmi->fb + 3) & ~3) * 4;
    const size_t xs_bytes = (size_t)3 * P.sc * P.sb * 32 * 4;
    // the x-contracted rows when two blocks per SM still fit
    P.xs = base_smem + xs_bytes <= 100 * 1024;
    const size_t smem = base_smem + (P.xs ? xs_bytes : 0);
    const int threads = 32 * ws->walk_obj.ty;
    const bool trial = grad != nullptr;
    auto kernel = P.flo_diag ? (trial ? (P.xs ? k_objective<true, true, true> : k_objective<true, false, true>)
                                      : (P.xs ? k_objective<false, true, true> : k_objective<false, false, true>))
                             : (trial ? (P.xs ? k_objective<true, true, false> : k_objective<true, false, false>)
                                      : (P.xs ? k_objective<false, true, false> : k_objective<false, false, false>));
    int grid = 0;
    NRB_TRY(persistent_grid(kernel, threads, smem, P.nitems, grid, ws->walk_obj.resident));
    // algorithmic bytes: reference + floating (+ mask) per voxel, the grid once
    const double nv = (double)P.nx * P.ny * P.nz;
    const double bytes = nv * (mask ? 12.0 : 8.0) + 12.0 * (double)P.cnv;
    cudaError_t e;
    {
        KernelTimer timer(TK_OBJECTIVE, bytes, st);
        e = launch_pdl(trial, kernel, dim3(grid), dim3(threads), smem, st, P, ref, flo, mask, cpp, nmi->hist, grad,
                       step);
    }
    NRB_CUDA(e);
    NRB_LAUNCHED("k_objective");
    return NRB_OK;
}

nrb_status launch_fused_gradient(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g,
                                 const float *ref, const float *flo, const int32_t *mask,
                                 const float *cpp, float padding, double weight, float *vgrad,
                                 cudaStream_t st, const OptState *sel, int flo_margin) {
    WalkParams P = make_params(ws->walk_grad, g, padding, nmi->rb, nmi->fb);
    set_floating_margin(P, flo_margin);
    P.ftex = flo_margin >= 2 ? ws->flo_tex : 0ull;
    // an FP32 copy of the log table rides in shared memory when it fits (64 bins: 19 KB,
    // 128 bins: 70 KB); larger tables use the FP64 window on the global table
    const size_t log_bytes = (size_t)nmi->total * sizeof(float);
    P.log_in_smem = log_bytes <= 96 * 1024;
    const size_t smem = walk_smem_bytes(ws->walk_grad) + (P.log_in_smem ? log_bytes : 0);
    const int threads = 32 * ws->walk_grad.ty;
    int grid = 0;
    auto kernel = P.flo_diag ? (P.log_in_smem ? k_gradient<true, true> : k_gradient<false, true>)
                             : (P.log_in_smem ? k_gradient<true, false> : k_gradient<false, false>);
    NRB_TRY(persistent_grid(kernel, threads, smem, P.nitems, grid, ws->walk_grad.resident));
    // algorithmic bytes: reference + floating (+ mask) read, voxel gradient written, grid once
    const double nv = (double)P.nx * P.ny * P.nz;
    const double bytes = nv * (mask ? 24.0 : 20.0) + 12.0 * (double)P.cnv;
    {
        KernelTimer timer(TK_GRADIENT, bytes, st);
        kernel<<<grid, threads, smem, st>>>(P, ref, flo, mask, cpp, nmi->logt, nmi->last, nmi->logt2, nmi->last2, sel,
                                            weight, vgrad);
    }
    NRB_LAUNCHED("k_gradient");
    return NRB_OK;
}

// ---- walk autotuner ---------------------------------------------------------------------------
namespace {

struct TuneKey {
    int rd[3], cd[3], gs[3];  // reference dims, grid dims, grid spacing in 1/1000 voxel
    int rb, fb, mask, margin, tex;
    bool operator<(const TuneKey& o) const {
        return std::memcmp(this, &o, sizeof(TuneKey)) < 0;
    }
};

struct TuneEntry {
    WalkPlan obj, grad;              // fastest measured
    WalkPlan obj_batch, grad_batch;  // fastest with the batched kernels' block shapes
    float obj_us = 0, grad_us = 0, obj_model_us = 0, grad_model_us = 0;
    int candidates = 0;
};

std::mutex g_tune_mu;
std::map<TuneKey, TuneEntry> g_tune;

TuneKey tune_key(const nrb_geometry *g, const nrb_nmi *nmi, const int32_t *mask, int margin, unsigned long long tex) {
    TuneKey k;
    std::memset(&k, 0, sizeof(k));
    for (int d = 0; d < 3; ++d) {
        k.rd[d] = g->ref_dim[d];
        k.cd[d] = g->cpp_dim[d];
        k.gs[d] = (int)lrintf(1000.f * g->cpp_pixdim[d] / g->ref_pixdim[d]);
    }
    k.rb = nmi->rb;
    k.fb = nmi->fb;
    k.mask = mask != nullptr;
    k.margin = margin > 0;
    k.tex = tex != 0;
    return k;
}

// mean device time of `reps` launches after one untimed launch; +inf if a launch fails
template <typename F>
float time_launch(F launch, cudaStream_t st, int reps) {
    cudaEvent_t a = nullptr, b = nullptr;
    float ms = INFINITY;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
        cudaGetLastError();
        if (a) cudaEventDestroy(a);
        return ms;
    }
    bool ok = launch() == NRB_OK && cudaEventRecord(a, st) == cudaSuccess;
    for (int r = 0; ok && r < reps; ++r) ok = launch() == NRB_OK;
    if (ok && cudaEventRecord(b, st) == cudaSuccess && cudaEventSynchronize(b) == cudaSuccess &&
        cudaEventElapsedTime(&ms, a, b) == cudaSuccess) {
        ms = ms * 1000.f / (float)reps;
    } else {
        ms = INFINITY;
        cudaGetLastError();
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

}  // namespace

bool autotune_lookup(nrb_workspace *ws, const nrb_nmi *nmi, const int32_t *mask, int flo_margin, bool batched) {
    const TuneKey k = tune_key(&ws->g, nmi, mask, flo_margin, ws->flo_tex);
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune.find(k);
    if (it == g_tune.end()) return false;
    ws->walk_obj = batched ? it->second.obj_batch : it->second.obj;
    ws->walk_grad = batched ? it->second.grad_batch : it->second.grad;
    return true;
}

nrb_status autotune_walks(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g, const float *ref, const float *flo,
                          const int32_t *mask, const float *cpp, float padding, int flo_margin, float *vgrad,
                          cudaStream_t st) {
    if (autotune_lookup(ws, nmi, mask, flo_margin, false)) return NRB_OK;
    const TuneKey key = tune_key(g, nmi, mask, flo_margin, ws->flo_tex);
    const WalkPlan obj0 = ws->walk_obj, grad0 = ws->walk_grad;
    constexpr int kChunks = 3, kReps = 3;
    const int sms = sm_count();
    TuneEntry e;
    // objective: two block heights, the model's best z-chunks, the occupancy limit or one block
    // per SM
    float best = INFINITY, best_batch = INFINITY;
    for (int ty : { TY_OBJECTIVE / 2, TY_OBJECTIVE }) {
        for (const WalkPlan& c : plan_walk_candidates(g, ty, objective_slots, OBJ_PLAN_EXTRA, 4, 6, kChunks)) {
            for (int resident : { 0, sms }) {
                WalkPlan w = c;
                w.resident = resident;
                ws->walk_obj = w;
                const float us = time_launch([&] {
                    return launch_fused_objective(ws, nmi, g, ref, flo, mask, cpp, padding, st, nullptr, nullptr,
                                                  flo_margin);
                }, st, kReps);
                ++e.candidates;
                if (ty == obj0.ty && resident == 0 && c.zchunk == obj0.zchunk) e.obj_model_us = us;
                if (us < best) { best = us; e.obj = w; }
                if (ty == TY_OBJECTIVE && resident == 0 && us < best_batch) { best_batch = us; e.obj_batch = w; }
            }
        }
    }
    e.obj_us = best;
    // the candidates' histogram counts go; the counts stay zero between evaluations
    NRB_CUDA(cudaMemsetAsync(nmi->hist, 0, (size_t)nmi->rb * nmi->fb * sizeof(uint32_t), st));
    best = best_batch = INFINITY;
    for (int ty : { TY_GRADIENT / 2, TY_GRADIENT }) {
        for (const WalkPlan& c : plan_walk_candidates(g, ty, gradient_slots, GRAD_PLAN_EXTRA, 4, 4, kChunks)) {
            for (int resident : { 0, 2 * sms }) {
                WalkPlan w = c;
                w.resident = resident;
                ws->walk_grad = w;
                const float us = time_launch([&] {
                    return launch_fused_gradient(ws, nmi, g, ref, flo, mask, cpp, padding, 1.0, vgrad, st, nullptr,
                                                 flo_margin);
                }, st, kReps);
                ++e.candidates;
                if (ty == grad0.ty && resident == 0 && c.zchunk == grad0.zchunk) e.grad_model_us = us;
                if (us < best) { best = us; e.grad = w; }
                if (ty == TY_GRADIENT && resident == 0 && us < best_batch) { best_batch = us; e.grad_batch = w; }
            }
        }
    }
    e.grad_us = best;
    if (!std::isfinite(e.obj_us) || !std::isfinite(e.grad_us) || e.obj_batch.ty == 0 || e.grad_batch.ty == 0) {
        ws->walk_obj = obj0;  // nothing measurable: keep the model's plans, record nothing
        ws->walk_grad = grad0;
        cudaGetLastError();
        return NRB_OK;
    }
    ws->walk_obj = e.obj;
    ws->walk_grad = e.grad;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune.emplace(key, e);
    return NRB_OK;
}

}  // namespace nrb

extern "C" int nrb_autotune_entries(nrb_walk_entry *out, int capacity) {
    std::lock_guard<std::mutex> lock(nrb::g_tune_mu);
    int i = 0;
    for (const auto& kv : nrb::g_tune) {
        if (out && i < capacity) {
            nrb_walk_entry& o = out[i];
            const nrb::TuneKey& k = kv.first;
            const nrb::TuneEntry& e = kv.second;
            for (int d = 0; d < 3; ++d) {
                o.ref_dim[d] = k.rd[d];
                o.cpp_dim[d] = k.cd[d];
            }
            o.bins[0] = k.rb - 4;
            o.bins[1] = k.fb - 4;
            o.obj_ty = e.obj.ty;
            o.obj_zchunk = e.obj.zchunk;
            o.obj_resident = e.obj.resident;
            o.obj_us = e.obj_us;
            o.obj_model_us = e.obj_model_us;
            o.grad_ty = e.grad.ty;
            o.grad_zchunk = e.grad.zchunk;
            o.grad_resident = e.grad.resident;
            o.grad_us = e.grad_us;
            o.grad_model_us = e.grad_model_us;
            o.candidates = e.candidates;
        }
        ++i;
    }
    return i;
}

extern "C" void nrb_autotune_clear(void) {
    std::lock_guard<std::mutex> lock(nrb::g_tune_mu);
    nrb::g_tune.clear();
}

namespace nrb {

nrb_status launch_nmi_finalize(nrb_nmi *nmi, const double *be_partials, int n_be_partials,
                               int64_t cpp_nvox3, double sim_weight, double be_weight,
                               nrb_objective *obj, cudaStream_t st, OptState *ctl,
                               cudaGraphConditionalHandle line, float *acc_best, const float *acc_grad,
                               long long acc_n) {
    const int rpc = (nmi->fb + FIN_CLUSTER - 1) / FIN_CLUSTER;
    const size_t smem = (size_t)(2 * rpc + 2) * nmi->rb * sizeof(double);
    NRB_CUDA(cudaFuncSetAttribute(k_nmi_finalize, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    KernelTimer timer(TK_FINALIZE, (double)nmi->rb * nmi->fb * 8 + (double)nmi->total * 16, st);
    FinArgs A;
    A.rb = nmi->rb;
    A.fb = nmi->fb;
    A.hist = nmi->hist;
    A.pro0 = nmi->pro;
    A.logt0 = nmi->logt;
    A.last0 = nmi->last;
    A.pro1 = nmi->pro2;
    A.logt1 = nmi->logt2;
    A.last1 = nmi->last2;
    A.be_partials = be_partials;
    A.n_be = n_be_partials;
    A.be_norm = (double)cpp_nvox3;
    A.sim_weight = sim_weight;
    A.be_weight = be_weight;
    A.obj = obj;
    A.ctl = ctl;
    A.acc_best = acc_best;
    A.acc_grad = acc_grad;
    A.acc_n = acc_n;
    NRB_CUDA(launch_pdl(ctl != nullptr, k_nmi_finalize, dim3(FIN_CLUSTER), dim3(FIN_CTA_THREADS), smem, st, A, line));
    NRB_LAUNCHED("k_nmi_finalize");
    return NRB_OK;
}

// ---- batched levels: walks, launch shapes, launches ----------------------------------------
nrb_status batch_walks(nrb_workspace *ws, const nrb_nmi *nmi, const nrb_geometry *g, float padding, int flo_margin,
                       WalkParams& wo, WalkParams& wg) {
    wo = make_params(ws->walk_obj, g, padding, nmi->rb, nmi->fb);
    set_floating_margin(wo, flo_margin);
    wg = make_params(ws->walk_grad, g, padding, nmi->rb, nmi->fb);
    set_floating_margin(wg, flo_margin);
    wo.ftex = wg.ftex = flo_margin >= 2 ? ws->flo_tex : 0ull;
    wg.log_in_smem = (size_t)nmi->total * sizeof(float) <= 96 * 1024;
    return NRB_OK;
}

nrb_status batch_plan(std::vector<BatchPair>& pairs, BatchLaunch& L) {
    L = BatchLaunch{};
    L.npairs = (int)pairs.size();
    if (L.npairs < 1 || L.npairs > BATCH_MAX_PAIRS)
        return fail(NRB_ERR_INVALID, "batched level: 1 to " + std::to_string(BATCH_MAX_PAIRS) + " pairs");
    size_t base = 0, xs = 0, gsm = 0;
    bool diag = true, f32 = true;
    int rb = pairs[0].rb, fb = pairs[0].fb;
    for (const BatchPair& b : pairs) {
        if (b.rb != rb || b.fb != fb) return fail(NRB_ERR_INVALID, "batched level: every pair needs the same bins");
        const size_t cp_o = (size_t)3 * b.wo.sa * b.wo.sb * b.wo.sc;
        base = std::max(base, (cp_o + 4 + (size_t)walk_table_floats(b.wo.zchunk)) * 4 + 16 +
                                  (size_t)((rb * fb + 3) & ~3) * 4);
        xs = std::max(xs, (size_t)3 * b.wo.sc * b.wo.sb * 32 * 4);
        const size_t cp_g = (size_t)3 * b.wg.sa * b.wg.sb * b.wg.sc;
        gsm = std::max(gsm, (cp_g + 4 + (size_t)walk_table_floats(b.wg.zchunk)) * 4 + 16);
        diag = diag && b.wo.flo_diag;
        f32 = f32 && b.wg.log_in_smem;
    }
    L.obj_xs = base + xs <= 100 * 1024;
    L.obj_diag = diag;
    L.obj_smem = base + (L.obj_xs ? xs : 0);
    L.grad_f32 = f32;
    L.grad_diag = diag;
    L.grad_smem = gsm + (f32 ? (size_t)(rb * fb + rb + fb) * sizeof(float) : 0);
    const int rpc = (fb + FIN_CLUSTER - 1) / FIN_CLUSTER;
    L.fin_smem = (size_t)(2 * rpc + 2) * rb * sizeof(double);
    for (size_t i = 0; i < pairs.size(); ++i) {
        BatchPair& b = pairs[i];
        b.wo.xs = L.obj_xs;
        b.wg.log_in_smem = f32;
        BatchObjEntry& o = L.obj_table.e[i];
        o.P = b.wo;
        o.ref = b.ref;
        o.flo = b.flo;
        o.best = b.best;
        o.grad = b.grad;
        o.hist = b.hist;
        BatchGradEntry& g = L.grad_table.e[i];
        g.P = b.wg;
        g.ref = b.ref;
        g.flo = b.flo;
        g.best = b.best;
        g.vgrad = b.vgrad;
        g.logt0 = b.logt0;
        g.logt1 = b.logt1;
        g.last0 = b.last0;
        g.last1 = b.last1;
    }
    auto ko = L.obj_diag ? (L.obj_xs ? k_b_objective<true, true> : k_b_objective<false, true>)
                         : (L.obj_xs ? k_b_objective<true, false> : k_b_objective<false, false>);
    auto kg = L.grad_diag ? (L.grad_f32 ? k_b_gradient<true, true> : k_b_gradient<false, true>)
                          : (L.grad_f32 ? k_b_gradient<true, false> : k_b_gradient<false, false>);
    int per = 0;
    NRB_CUDA(cudaFuncSetAttribute(ko, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    NRB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, ko, 32 * TY_OBJECTIVE, L.obj_smem));
    L.obj_grid = std::max(1, per) * sm_count();
    NRB_CUDA(cudaFuncSetAttribute(kg, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    NRB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kg, 32 * TY_GRADIENT, L.grad_smem));
    L.grad_grid = std::max(1, per) * sm_count();
    NRB_CUDA(cudaFuncSetAttribute(k_b_finalize, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.fin_smem));
    return NRB_OK;
}

nrb_status launch_batch_objective(const BatchPair *d_pairs, const OptState *states, const BatchLaunch& L,
                                  cudaStream_t st, double bytes) {
    KernelTimer timer(TK_OBJECTIVE, bytes, st);
    auto ko = L.obj_diag ? (L.obj_xs ? k_b_objective<true, true> : k_b_objective<false, true>)
                         : (L.obj_xs ? k_b_objective<true, false> : k_b_objective<false, false>);
    ko<<<L.obj_grid, 32 * TY_OBJECTIVE, L.obj_smem, st>>>(L.obj_table, states, L.npairs);
    NRB_CUDA(cudaGetLastError());
    NRB_LAUNCHED("k_b_objective");
    return NRB_OK;
}

nrb_status launch_batch_gradient(const BatchPair *d_pairs, const OptState *states, const BatchLaunch& L,
                                 cudaStream_t st, double bytes) {
    KernelTimer timer(TK_GRADIENT, bytes, st);
    auto kg = L.grad_diag ? (L.grad_f32 ? k_b_gradient<true, true> : k_b_gradient<false, true>)
                          : (L.grad_f32 ? k_b_gradient<true, false> : k_b_gradient<false, false>);
    kg<<<L.grad_grid, 32 * TY_GRADIENT, L.grad_smem, st>>>(L.grad_table, states, L.npairs);
    NRB_CUDA(cudaGetLastError());
    NRB_LAUNCHED("k_b_gradient");
    return NRB_OK;
}

nrb_status launch_batch_finalize(const BatchPair *d_pairs, OptState *states, BatchCtl *bctl, const BatchLaunch& L,
                                 bool in_graph, cudaGraphConditionalHandle grad_if, cudaGraphConditionalHandle outer,
                                 cudaStream_t st) {
    KernelTimer timer(TK_FINALIZE, 0.0, st);
    NRB_CUDA(launch_pdl(in_graph, k_b_finalize, dim3(FIN_CLUSTER * L.npairs), dim3(FIN_CTA_THREADS), L.fin_smem, st,
                        d_pairs, states, L.npairs, bctl, in_graph ? 1 : 0, grad_if, outer));
    NRB_LAUNCHED("k_b_finalize");
    return NRB_OK;
}

// ---- floating-image textures ---------------------------------------------------------------
namespace {
std::mutex g_tex_mu;
std::vector<FloTexture> g_tex_free;  // unused arrays, any device
size_t g_tex_free_bytes = 0;
constexpr size_t kTexPoolKeepBytes = size_t(4) << 30;

size_t tex_bytes(const FloTexture& t) { return (size_t)t.width * t.height * t.layers * sizeof(float); }

void tex_destroy(FloTexture& t) {
    int cur = -1;
    cudaGetDevice(&cur);
    if (t.device >= 0 && t.device != cur) cudaSetDevice(t.device);
    if (t.tex) cudaDestroyTextureObject((cudaTextureObject_t)t.tex);
    if (t.arr) cudaFreeArray(t.arr);
    if (t.device >= 0 && t.device != cur) cudaSetDevice(cur);
    cudaGetLastError();
    t = FloTexture{};
}
}  // namespace

nrb_status flo_texture_acquire(int width, int height, int layers, FloTexture& out) {
    out = FloTexture{};
    if (width < 1 || height < 1 || layers < 1 || width > 32768 || height > 32768 || layers > 2048)
        return fail(NRB_ERR_UNSUPPORTED, "floating texture: extent outside a layered array's limits");
    int dev = 0;
    NRB_CUDA(cudaGetDevice(&dev));
    {
        // the smallest unused array of this device that holds the extent
        std::lock_guard<std::mutex> lock(g_tex_mu);
        int best = -1;
        for (int i = 0; i < (int)g_tex_free.size(); ++i) {
            const FloTexture& t = g_tex_free[i];
            if (t.device == dev && t.width >= width && t.height >= height && t.layers >= layers &&
                (best < 0 || tex_bytes(t) < tex_bytes(g_tex_free[best])))
                best = i;
        }
        if (best >= 0) {
            out = g_tex_free[best];
            g_tex_free_bytes -= tex_bytes(out);
            g_tex_free.erase(g_tex_free.begin() + best);
            return NRB_OK;
        }
    }
    FloTexture t;
    t.device = dev;
    t.width = width;
    t.height = height;
    t.layers = layers;
    const cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
    NRB_CUDA(cudaMalloc3DArray(&t.arr, &cd, make_cudaExtent(width, height, layers), cudaArrayLayered));
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = t.arr;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaTextureObject_t obj = 0;
    const cudaError_t e = cudaCreateTextureObject(&obj, &rd, &td, nullptr);
    if (e != cudaSuccess) {
        cudaFreeArray(t.arr);
        return check_cuda(e, "cudaCreateTextureObject");
    }
    t.tex = (unsigned long long)obj;
    out = t;
    return NRB_OK;
}

void flo_texture_release(FloTexture& t) {
    if (!t.arr) return;
    std::lock_guard<std::mutex> lock(g_tex_mu);
    g_tex_free.push_back(t);
    g_tex_free_bytes += tex_bytes(t);
    // over the cap: free the largest unused arrays first
    while (g_tex_free_bytes > kTexPoolKeepBytes && !g_tex_free.empty()) {
        int big = 0;
        for (int i = 1; i < (int)g_tex_free.size(); ++i)
            if (tex_bytes(g_tex_free[i]) > tex_bytes(g_tex_free[big])) big = i;
        g_tex_free_bytes -= tex_bytes(g_tex_free[big]);
        tex_destroy(g_tex_free[big]);
        g_tex_free.erase(g_tex_free.begin() + big);
    }
    t = FloTexture{};
}

nrb_status flo_texture_upload(const FloTexture& t, const float *src, int width, int height, int layers,
                              cudaStream_t st) {
    if (width > t.width || height > t.height || layers > t.layers)
        return fail(NRB_ERR_INVALID, "floating texture: volume larger than the array");
    cudaMemcpy3DParms p = {};
    p.srcPtr = make_cudaPitchedPtr(const_cast<float *>(src), (size_t)width * sizeof(float), width, height);
    p.dstArray = t.arr;
    p.extent = make_cudaExtent(width, height, layers);
    p.kind = cudaMemcpyDeviceToDevice;
    NRB_CUDA(cudaMemcpy3DAsync(&p, st));
    return NRB_OK;
}

}  // namespace nrb

using namespace nrb;

extern "C" nrb_status nrb_get_deformation_field(const nrb_geometry *g, const float *cpp,
                                                const int32_t *mask, float *def, void *stream) {
    if (!g || !cpp || !def) return fail(NRB_ERR_INVALID, "nrb_get_deformation_field: null pointer");
    NRB_TRY(validate_geometry(g));
    const WalkPlan W = plan_walk(g, TY_DEFORMATION, deformation_slots, 0);
    const WalkParams P = make_params(W, g, 0.f, 0, 0);
    const size_t smem = walk_smem_bytes(W);
    int grid = 0;
    NRB_TRY(persistent_grid(k_deformation, 32 * W.ty, smem, P.nitems, grid));
    k_deformation<<<grid, 32 * W.ty, smem, as_stream(stream)>>>(P, mask, cpp, def);
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
    const int grid = (int)std::min<long long>((nv + threads - 1) / threads, 64LL * sm_count());
    const Mat34 M = to_mat34(g->flo_ijk);
    const float *m = g->flo_ijk;
    const int diag = m[1] == 0.f && m[2] == 0.f && m[4] == 0.f && m[6] == 0.f && m[8] == 0.f && m[9] == 0.f;
    if (grad)
        k_resample<true><<<grid, threads, 0, as_stream(stream)>>>(nv, g->flo_dim[0], g->flo_dim[1], g->flo_dim[2], M,
                                                                  diag, pad, flo, def, mask, out);
    else
        k_resample<false><<<grid, threads, 0, as_stream(stream)>>>(nv, g->flo_dim[0], g->flo_dim[1], g->flo_dim[2], M,
                                                                   diag, pad, flo, def, mask, out);
    NRB_LAUNCHED("k_resample");
    return NRB_OK;
}

extern "C" nrb_status nrb_resample_image(const nrb_geometry *g, const float *flo, const float *def,
                                         const int32_t *mask, float padding, float *warped,
                                         void *stream) {
    return resample_common(g, flo, def, mask, padding, warped, false, stream);
}

namespace nrb {
nrb_status resample_order(const nrb_geometry *g, const float *flo, const float *def, const int32_t *mask,
                          int order, float padding, float *warped, cudaStream_t st) {
    if (!g || !flo || !def || !warped) return fail(NRB_ERR_INVALID, "resample: null pointer");
    if (order != 0 && order != 1 && order != 3)
        return fail(NRB_ERR_UNSUPPORTED, "resample: interpolation order must be 0 (nearest), 1 (linear) or 3 (cubic spline)");
    const long long nv = nvox(g->ref_dim);
    if (nv <= 0) return fail(NRB_ERR_INVALID, "resample: empty reference");
    const int threads = 256;
    const int grid = (int)std::min<long long>((nv + threads - 1) / threads, 64LL * sm_count());
    const Mat34 M = to_mat34(g->flo_ijk);
    const int fx = g->flo_dim[0], fy = g->flo_dim[1], fz = g->flo_dim[2];
    if (order == 0)
        k_resample_order<0><<<grid, threads, 0, st>>>(nv, fx, fy, fz, M, padding, flo, def, mask, warped);
    else if (order == 1)
        k_resample_order<1><<<grid, threads, 0, st>>>(nv, fx, fy, fz, M, padding, flo, def, mask, warped);
    else
        k_resample_order<3><<<grid, threads, 0, st>>>(nv, fx, fy, fz, M, padding, flo, def, mask, warped);
    NRB_LAUNCHED("k_resample_order");
    return NRB_OK;
}
}  // namespace nrb

extern "C" nrb_status nrb_resample_image_order(const nrb_geometry *g, const float *flo, const float *def,
                                               const int32_t *mask, int order, float padding, float *warped,
                                               void *stream) {
    return resample_order(g, flo, def, mask, order, padding, warped, as_stream(stream));
}

extern "C" nrb_status nrb_f3d_warped_image(const nrb_geometry *g, const float *flo, const float *cpp, int order,
                                           float padding, float *warped, void *stream) {
    if (!g || !flo || !cpp || !warped) return fail(NRB_ERR_INVALID, "nrb_f3d_warped_image: null pointer");
    NRB_TRY(validate_geometry(g));
    if (order != 0 && order != 1 && order != 3)
        return fail(NRB_ERR_UNSUPPORTED, "nrb_f3d_warped_image: interpolation order must be 0, 1 or 3");
    const WalkPlan W = plan_walk(g, TY_DEFORMATION, deformation_slots, 0);
    const WalkParams P = make_params(W, g, padding, 0, 0);
    const size_t smem = walk_smem_bytes(W);
    auto kernel = order == 0 ? k_warp_order<0> : order == 1 ? k_warp_order<1> : k_warp_order<3>;
    int grid = 0;
    NRB_TRY(persistent_grid(kernel, 32 * W.ty, smem, P.nitems, grid));
    kernel<<<grid, 32 * W.ty, smem, as_stream(stream)>>>(P, cpp, flo, warped);
    NRB_LAUNCHED("k_warp_order");
    return NRB_OK;
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

namespace nrb {
// fp64: the FP64 window whatever the table size (the F3D2 driver keeps it, so that its
// trajectory follows reg_f3d2's); otherwise the FP32 window when the table fits
nrb_status nmi_voxel_gradient(nrb_nmi *nmi, const nrb_geometry *g, const float *ref, const float *warped,
                              const float *warped_grad, const int32_t *mask, double weight, float *vgrad,
                              cudaStream_t st, bool fp64) {
    const long long nv = nvox(g->ref_dim);
    const int threads = 256;
    const int grid = (int)std::min<long long>((nv + threads - 1) / threads, 16LL * sm_count());
    // the FP32 window when the log table fits in shared memory (64 bins: 19 KB, 128 bins: 70 KB)
    const size_t log_bytes = (size_t)nmi->total * sizeof(float);
    if (!fp64 && log_bytes <= 96 * 1024) {
        NRB_CUDA(cudaFuncSetAttribute(k_nmi_voxel_gradient<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)log_bytes));
        k_nmi_voxel_gradient<true><<<grid, threads, log_bytes, st>>>(nv, nmi->rb, nmi->fb, ref, warped, warped_grad,
                                                                     mask, nmi->logt, nmi->last, weight, vgrad);
    } else {
        k_nmi_voxel_gradient<false><<<grid, threads, 0, st>>>(nv, nmi->rb, nmi->fb, ref, warped, warped_grad, mask,
                                                              nmi->logt, nmi->last, weight, vgrad);
    }
    NRB_CUDA(cudaGetLastError());
    NRB_LAUNCHED("k_nmi_voxel_gradient");
    return NRB_OK;
}
}  // namespace nrb

extern "C" nrb_status nrb_nmi_voxel_gradient(nrb_nmi *nmi, const nrb_geometry *g, const float *ref,
                                             const float *warped, const float *warped_grad,
                                             const int32_t *mask, double weight, float *vgrad,
                                             void *stream) {
    if (!nmi || !g || !ref || !warped || !warped_grad || !vgrad)
        return fail(NRB_ERR_INVALID, "nrb_nmi_voxel_gradient: null pointer");
    return nmi_voxel_gradient(nmi, g, ref, warped, warped_grad, mask, weight, vgrad, as_stream(stream), false);
}
