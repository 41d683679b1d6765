// Node-grid and reduction kernels of the F3D gradient path, the voxel->node convolution, the
// image pyramid and the workspace that sizes their scratch buffers.
//
// Every reduction writes a fixed number of per-block partials and combines them in a fixed
// order, so each result is identical from run to run whatever the device's SM count.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <mutex>
#include <vector>

#include "nrb_state.cuh"

namespace nrb {

// ---------------------------------------------------------------------------------------------
// bending energy
// ---------------------------------------------------------------------------------------------
// Second-derivative stencils at the nodes in the 27-point (c, b, a) order of
// set_second_order_bspline_basis_values (reg-lib/cpu/_reg_splineBasis.cpp:291-455). The
// reference tabulates the exact values rounded to 6 decimals; the same rounding is applied
// here to B(+-1) = 1/6, B(0) = 2/3, B'(+-1) = +-1/2, B'(0) = 0, B''(+-1) = 1, B''(0) = -2.
static BeBasis make_be_basis() {
    const double B[3] = { 1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0 };
    const double D[3] = { -0.5, 0.0, 0.5 };
    const double S[3] = { 1.0, -2.0, 1.0 };
    auto r6 = [](double x) { return (float)(std::round(x * 1e6) / 1e6); };
    BeBasis b;
    int i = 0;
    for (int c = 0; c < 3; ++c)
        for (int bb = 0; bb < 3; ++bb)
            for (int a = 0; a < 3; ++a, ++i) {
                b.v[0][i] = r6(S[a] * B[bb] * B[c]);
                b.v[1][i] = r6(B[a] * S[bb] * B[c]);
                b.v[2][i] = r6(B[a] * B[bb] * S[c]);
                b.v[3][i] = r6(D[a] * D[bb] * B[c]);
                b.v[4][i] = r6(B[a] * D[bb] * D[c]);
                b.v[5][i] = r6(D[a] * B[bb] * D[c]);
            }
    return b;
}

static const BeBasis& be_basis() {
    static const BeBasis b = make_be_basis();
    return b;
}

__device__ double block_sum_d(double v, double *red) {
    const int tid = threadIdx.x;
    red[tid] = v;
    __syncthreads();
    for (int s = NRB_RED_THREADS / 2; s > 0; s >>= 1) {
        if (tid < s) red[tid] += red[tid + s];
        __syncthreads();
    }
    return red[0];
}

// reg_spline_approxBendingEnergyValue3D (reg-lib/cpu/_reg_localTrans_regul.cpp:72-153): per
// interior node the 6 second derivatives of each component from 27-point stencils of the
// positions, summed squares (cross terms doubled) accumulated in double. The stencil sums use
// the reference's order without contraction: each node's terms are bit-identical to the CPU's.
// grad/step (optional): the positions are the line search's trial values cpp - cur_len * grad
//
// Three threads per node, one per component (threads k * NRB_RED_THREADS + j of a block), so 27
// loads per thread are in flight and three times as many warps hide their latency. Node lane j
// (component 0) adds the other components' terms in the reference's order and accumulates its
// nodes in the grid-stride order of a one-thread-per-node loop; the block sum is the same tree
// as block_sum_d over the NRB_RED_THREADS node lanes, so every partial is unchanged bit for bit.
__global__ void __launch_bounds__(3 * NRB_RED_THREADS, 2)
k_be_value(int cx, int cy, int cz, const float *__restrict__ cpp, BeBasis B,
           double *__restrict__ partials, const float *__restrict__ grad, const OptState *__restrict__ step) {
    __shared__ double red[NRB_RED_THREADS];
    __shared__ BeTerms other[2][NRB_RED_THREADS];  // components 1 and 2 of the lane's node
    const float scale = grad ? -step->cur_len : 0.f;
    const int j = threadIdx.x % NRB_RED_THREADS, k = threadIdx.x / NRB_RED_THREADS;
    const int ix = cx - 2, iy = cy - 2, iz = cz - 2;
    const long long ni = (ix > 0 && iy > 0 && iz > 0) ? (long long)ix * iy * iz : 0;
    double acc = 0;
    for (long long base = blockIdx.x * (long long)NRB_RED_THREADS; base < ni; base += (long long)gridDim.x * NRB_RED_THREADS) {
        const long long n = base + j;
        BeTerms t{ 0.f, 0.f, 0.f, 0.f };
        if (n < ni) t = be_node_component<true>(cx, cy, cz, ix, iy, cpp, B, grad, scale, n, k);
        if (k > 0) other[k - 1][j] = t;
        __syncthreads();
        if (k == 0 && n < ni) {
            double s = be_add_component(0.0, t, 0);
            s = be_add_component(s, other[0][j], 1);
            acc += be_add_component(s, other[1][j], 2);
        }
        __syncthreads();  // `other` is rewritten by the next round
    }
    if (k == 0) red[j] = acc;
    __syncthreads();
    for (int s = NRB_RED_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

__global__ void k_be_sum(const double *__restrict__ partials, int n, double norm,
                         nrb_objective *__restrict__ obj) {
    __shared__ double red[NRB_RED_THREADS];
    double a = 0;
    for (int i = threadIdx.x; i < n; i += NRB_RED_THREADS) a += partials[i];
    const double s = block_sum_d(a, red);
    if (threadIdx.x == 0) obj->be = s / norm;
}

// Node position on the identity grid, float arithmetic in the reference's order
// (reg_getDisplacementFromDeformation_3D, reg-lib/cpu/_reg_tools.cpp:2011-2022).
__device__ __forceinline__ float identity_pos(const Mat34& M, int k, int x, int y, int z) {
    const float *m = M.m + 4 * k;
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], (float)x), __fmul_rn(m[1], (float)y)),
                               __fmul_rn(m[2], (float)z)), m[3]);
}

// reg_spline_approxBendingEnergyGradient3D (reg-lib/cpu/_reg_localTrans_regul.cpp:286-451),
// first half: the 6 derivative values of component k of node n from zero-padded stencils of the
// displacements, cross terms doubled. Layout der[(3 * t + k) * nc + node].
__device__ __forceinline__ void be_node_derivatives_k(int cx, int cy, int cz, const Mat34& M,
                                                      const float *__restrict__ cpp, const BeBasis& B,
                                                      float *__restrict__ der, long long n, int k) {
    const long long nc = (long long)cx * cy * cz;
    const int x = (int)(n % cx);
    const int y = (int)((n / cx) % cy);
    const int z = (int)(n / ((long long)cx * cy));
    // row k of the grid matrix picked by selects (a runtime index into the parameter would copy
    // the matrix to local memory)
    float m[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) m[q] = k == 0 ? M.m[q] : (k == 1 ? M.m[4 + q] : M.m[8 + q]);
    float d[6];
#pragma unroll
    for (int t = 0; t < 6; ++t) d[t] = 0.f;
#pragma unroll
    for (int c = -1; c < 2; ++c)
#pragma unroll
        for (int b = -1; b < 2; ++b)
#pragma unroll
            for (int a = -1; a < 2; ++a) {
                const int i = 9 * (c + 1) + 3 * (b + 1) + (a + 1);
                const int X = x + a, Y = y + b, Z = z + c;
                if (X < 0 || Y < 0 || Z < 0 || X >= cx || Y >= cy || Z >= cz) continue;
                const long long idx = ((long long)Z * cy + Y) * cx + X;
                const float id = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], (float)X), __fmul_rn(m[1], (float)Y)),
                                                     __fmul_rn(m[2], (float)Z)), m[3]);  // identity_pos
                const float v = __fsub_rn(__ldg(&cpp[k * nc + idx]), id);
#pragma unroll
                for (int t = 0; t < 6; ++t) d[t] = __fadd_rn(d[t], __fmul_rn(B.v[t][i], v));
            }
#pragma unroll
    for (int t = 0; t < 3; ++t) der[(3 * t + k) * nc + n] = d[t];
#pragma unroll
    for (int t = 3; t < 6; ++t) der[(3 * t + k) * nc + n] = (float)(2.0 * (double)d[t]);
}

// one thread per (node, component): component k = blockIdx.y
__global__ void k_be_derivatives(int cx, int cy, int cz, Mat34 M, const float *__restrict__ cpp,
                                 BeBasis B, float *__restrict__ der) {
    const long long nc = (long long)cx * cy * cz;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nc;
         n += (long long)gridDim.x * blockDim.x)
        be_node_derivatives_k(cx, cy, cz, M, cpp, B, der, n, (int)blockIdx.y);
}

// second half: the same stencils applied to the derivative values of the 27 neighbours,
// grad += weight / #nodes * sum, for component k of node n: the sum runs over the neighbours
// in (z, y, x) order and the 6 derivative kinds within each, as for all components at once.
__device__ __forceinline__ void be_node_accumulate_k(int cx, int cy, int cz, const float *__restrict__ der,
                                                     const BeBasis& B, float ratio, float *__restrict__ grad,
                                                     long long n, int k) {
    const long long nc = (long long)cx * cy * cz;
    const int x = (int)(n % cx);
    const int y = (int)((n / cx) % cy);
    const int z = (int)(n / ((long long)cx * cy));
    float g = 0.f;
#pragma unroll
    for (int c = -1; c < 2; ++c)
#pragma unroll
        for (int b = -1; b < 2; ++b)
#pragma unroll
            for (int e = -1; e < 2; ++e) {
                const int a = 9 * (c + 1) + 3 * (b + 1) + (e + 1);
                const int X = x + e, Y = y + b, Z = z + c;
                if (X < 0 || Y < 0 || Z < 0 || X >= cx || Y >= cy || Z >= cz) continue;
                const long long j = ((long long)Z * cy + Y) * cx + X;
#pragma unroll
                for (int t = 0; t < 6; ++t) g = __fadd_rn(g, __fmul_rn(__ldg(&der[(3 * t + k) * nc + j]), B.v[t][a]));
            }
    grad[k * nc + n] = __fadd_rn(grad[k * nc + n], __fmul_rn(ratio, g));
}

// one thread per (node, component): component k = blockIdx.y
__global__ void k_be_accumulate(int cx, int cy, int cz, const float *__restrict__ der, BeBasis B,
                                float ratio, float *__restrict__ grad) {
    const long long nc = (long long)cx * cy * cz;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nc;
         n += (long long)gridDim.x * blockDim.x)
        be_node_accumulate_k(cx, cy, cz, der, B, ratio, grad, n, (int)blockIdx.y);
}

// ---------------------------------------------------------------------------------------------
// voxel -> node: cubic convolution evaluated only at the sampled voxels
// ---------------------------------------------------------------------------------------------
// Normalised convolution of one line at one sample: density = finite(value) (the reference's
// mask is all-active here), NaN at the sample itself stays NaN (_reg_tools.cpp:863-867, :1105).
template <typename Load>
__device__ __forceinline__ float conv_at(int s, int n, int R, const float *__restrict__ K, Load ld) {
    const float centre = ld(s);
    if (centre != centre) return centre;
    float num = 0.f, den = 0.f;
    const int k0 = max(0, s - R), k1 = min(n - 1, s + R);
    for (int k = k0; k <= k1; ++k) {
        const float v = ld(k);
        const float w = K[k - s + R];
        if (v == v) {
            num = fmaf(w, v, num);
            den += w;
        }
    }
    return num / den;
}

// pass along x: a block stages CONV_X_ROWS consecutive (y, z) rows of each component in shared
// memory (for a component those rows are one contiguous run of the volume, so the loads
// coalesce and many are in flight per thread), then evaluates the sampled outputs of all of them
constexpr int CONV_X_ROWS = 8, CONV_X_THREADS = 256;

// rows [rb * CONV_X_ROWS, ...) of the x pass; `rows` is the block's shared memory
// ([3][CONV_X_ROWS][nx] | kernel taps [2R + 1]); ends with every output of those rows written
__device__ __forceinline__ void conv_x_rows(int nx, int ny, int nz, const float *__restrict__ vg,
                                            const int *__restrict__ samples, int ns, const float *__restrict__ K,
                                            int R, float *__restrict__ out, long long rb, float *rows) {
    float *Ks = rows + 3 * CONV_X_ROWS * nx;
    const long long nv = (long long)nx * ny * nz;
    const long long nrow = (long long)ny * nz;
    const long long r0 = rb * CONV_X_ROWS;
    const int nr = (int)min((long long)CONV_X_ROWS, nrow - r0);
    const int run = nr * nx;
    int nan = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float *src = vg + c * nv + r0 * nx;
        float *dst = rows + c * CONV_X_ROWS * nx;
        for (int i = threadIdx.x; i < run; i += CONV_X_THREADS) {
            const float v = __ldg(src + i);
            nan |= v != v;
            dst[i] = v;
        }
    }
    for (int i = threadIdx.x; i < 2 * R + 1; i += CONV_X_THREADS) Ks[i] = K[i];
    // each sample's sum of in-row kernel weights (the same for every row without NaN), summed in
    // the order of the check-free loop below
    float *dens = Ks + 2 * R + 1;
    for (int j = threadIdx.x; j < ns; j += CONV_X_THREADS) {
        const int sj = samples[j];
        const int k0 = max(0, sj - R), k1 = min(nx - 1, sj + R);
        float den = 0.f;
        for (int k = k0; k <= k1; ++k) den += K[k - sj + R];
        dens[j] = den;
    }
    // rows without NaN (the fused gradient never writes one) take the check-free sum: the
    // same operations in the same order as conv_at when every tap counts
    const bool any_nan = __syncthreads_or(nan) != 0;
    if (ns <= 0) return;  // no sample on this axis: nothing to write
    // outputs (component c, row r < CONV_X_ROWS, sample j) in the order cr = c * CONV_X_ROWS + r,
    // then j; a thread steps by CONV_X_THREADS outputs with carried counters (no division per
    // output); rows beyond the block's last (r >= nr) are skipped
    int j = threadIdx.x % ns, cr = threadIdx.x / ns;
    const int dj = CONV_X_THREADS % ns, dcr = CONV_X_THREADS / ns;
    for (; cr < 3 * CONV_X_ROWS; cr += dcr) {
        const int c = cr / CONV_X_ROWS, r = cr % CONV_X_ROWS;
        if (r < nr) {
            const float *row = rows + cr * nx;
            const int sj = samples[j];
            float v;
            if (any_nan) {
                v = conv_at(sj, nx, R, Ks, [&](int k) { return row[k]; });
            } else {
                float num = 0.f;
                const int k0 = max(0, sj - R), k1 = min(nx - 1, sj + R);
                const float *w = Ks - sj + R;
#pragma unroll 4
                for (int k = k0; k <= k1; ++k) num = fmaf(w[k], row[k], num);
                v = num / dens[j];
            }
            out[(c * nrow + r0 + r) * ns + j] = v;
        }
        j += dj;
        if (j >= ns) {
            j -= ns;
            ++cr;
        }
    }
}

__global__ void __launch_bounds__(CONV_X_THREADS)
k_conv_x(int nx, int ny, int nz, const float *__restrict__ vg, const int *__restrict__ samples, int ns,
         const float *__restrict__ K, int R, float *__restrict__ out) {
    extern __shared__ float rows[];
    conv_x_rows(nx, ny, nz, vg, samples, ns, K, R, out, blockIdx.x, rows);
}

// pass along an outer axis of a [3][outer][len][inner] array at sampled positions of `len`:
// out[3][outer][ns][inner]
__device__ __forceinline__ void conv_strided_at(int outer, int len, int inner, const float *__restrict__ in,
                                                const int *__restrict__ samples, int ns, const float *__restrict__ K,
                                                int R, float *__restrict__ out, long long i) {
    {
        const int ii = (int)(i % inner);
        long long rest = i / inner;
        const int j = (int)(rest % ns);
        rest /= ns;
        const int o = (int)(rest % outer);
        const int c = (int)(rest / outer);
        const float *base = in + (((long long)c * outer + o) * len) * inner + ii;
        out[i] = conv_at(samples[j], len, R, K, [&](int k) { return __ldg(&base[(long long)k * inner]); });
    }
}

__global__ void k_conv_strided(int outer, int len, int inner, const float *__restrict__ in,
                               const int *__restrict__ samples, int ns, const float *__restrict__ K,
                               int R, float *__restrict__ out) {
    const long long total = 3LL * outer * ns * inner;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x)
        conv_strided_at(outer, len, inner, in, samples, ns, K, R, out, i);
}

// reg_voxelCentricToNodeCentric (reg-lib/cpu/_reg_localTrans.cpp:1616-1683): trilinear sample
// of the convolved gradient (taps outside the volume skipped), reorientation by the transpose
// of the floating ijk 3x3, weighting; overwrites the node gradient.
__device__ __forceinline__ void node_at(int cx, int cy, int cz, int nsx, int nsy, int nsz,
                                        const float *__restrict__ conv, const int *__restrict__ tsx,
                                        const float *__restrict__ wsx, const int *__restrict__ tsy,
                                        const float *__restrict__ wsy, const int *__restrict__ tsz,
                                        const float *__restrict__ wsz, const Mat34& R, float weight,
                                        float *__restrict__ node, long long n) {
    const long long nc = (long long)cx * cy * cz;
    const long long cs = (long long)nsz * nsy * nsx;
    {
        const int x = (int)(n % cx);
        const int y = (int)((n / cx) % cy);
        const int z = (int)(n / ((long long)cx * cy));
        float iv[3] = { 0.f, 0.f, 0.f };
        for (int c = 0; c < 2; ++c) {
            const int sz = tsz[2 * z + c];
            if (sz < 0) continue;
            const float wz = wsz[2 * z + c];
            for (int b = 0; b < 2; ++b) {
                const int sy = tsy[2 * y + b];
                if (sy < 0) continue;
                const float wy = wsy[2 * y + b];
                for (int a = 0; a < 2; ++a) {
                    const int sx = tsx[2 * x + a];
                    if (sx < 0) continue;
                    const float lw = __fmul_rn(__fmul_rn(wsx[2 * x + a], wy), wz);
                    const long long idx = ((long long)sz * nsy + sy) * nsx + sx;
                    iv[0] = fmaf(lw, conv[idx], iv[0]);
                    iv[1] = fmaf(lw, conv[cs + idx], iv[1]);
                    iv[2] = fmaf(lw, conv[2 * cs + idx], iv[2]);
                }
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const float ro = R.m[0 * 4 + d] * iv[0] + R.m[1 * 4 + d] * iv[1] + R.m[2 * 4 + d] * iv[2];
            node[d * nc + n] = ro * weight;
        }
    }
}

__global__ void k_nodes(int cx, int cy, int cz, int nsx, int nsy, int nsz,
                        const float *__restrict__ conv, const int *__restrict__ tsx,
                        const float *__restrict__ wsx, const int *__restrict__ tsy,
                        const float *__restrict__ wsy, const int *__restrict__ tsz,
                        const float *__restrict__ wsz, Mat34 R, float weight,
                        float *__restrict__ node) {
    const long long nc = (long long)cx * cy * cz;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nc;
         n += (long long)gridDim.x * blockDim.x)
        node_at(cx, cy, cz, nsx, nsy, nsz, conv, tsx, wsx, tsy, wsy, tsz, wsz, R, weight, node, n);
}

// ---------------------------------------------------------------------------------------------
// batched levels: the node-grid and node-convolution stages of every pair that needs them, with
// each pair's elements computed exactly as the plain kernels compute them
// ---------------------------------------------------------------------------------------------
// bending-energy value partials of every pair in INIT or LINE: work unit = one block of the plain
// k_be_value (same node range, three threads per node, same shared-memory tree), persistent
// blocks of 3 * NRB_RED_THREADS
__global__ void __launch_bounds__(3 * NRB_RED_THREADS, 2)
k_b_be_value(const BatchPair *__restrict__ pairs, const OptState *__restrict__ states, int npairs, BeBasis B) {
    __shared__ BatchList L;
    __shared__ double red[NRB_RED_THREADS];
    __shared__ BeTerms other[2][NRB_RED_THREADS];
    const int j = threadIdx.x % NRB_RED_THREADS, kc = threadIdx.x / NRB_RED_THREADS;
    batch_list_build(states, npairs, (1u << PH_INIT) | (1u << PH_LINE),
                     [&](int q, int& u, int& w) {
                         const BatchPair& b = pairs[q];
                         u = b.be_w > 0 ? b.n_be : 0;
                         w = 1;
                     }, L);
    int k = 0;
    for (long long u = blockIdx.x; u < L.total; u += gridDim.x) {
        while (L.pref[k + 1] <= u) ++k;
        const int p = L.pair[k], v = (int)(u - L.pref[k]);
        const BatchPair& P = pairs[p];
        const bool line = states[p].phase == PH_LINE;
        const float *grad = line ? P.grad : nullptr;
        const float scale = line ? -states[p].cur_len : 0.f;
        const int cx = P.cdim[0], cy = P.cdim[1], cz = P.cdim[2];
        const int ix = cx - 2, iy = cy - 2, iz = cz - 2;
        const long long ni = (ix > 0 && iy > 0 && iz > 0) ? (long long)ix * iy * iz : 0;
        double acc = 0;
        // the unit's bounds are the same for every thread of the block (one pair per unit)
        for (long long base = (long long)v * NRB_RED_THREADS; base < ni; base += (long long)P.n_be * NRB_RED_THREADS) {
            const long long n = base + j;
            BeTerms t{ 0.f, 0.f, 0.f, 0.f };
            if (n < ni) t = be_node_component<true>(cx, cy, cz, ix, iy, P.best, B, grad, scale, n, kc);
            if (kc > 0) other[kc - 1][j] = t;
            __syncthreads();
            if (kc == 0 && n < ni) {
                double s = be_add_component(0.0, t, 0);
                s = be_add_component(s, other[0][j], 1);
                acc += be_add_component(s, other[1][j], 2);
            }
            __syncthreads();
        }
        if (kc == 0) red[j] = acc;
        __syncthreads();
        for (int s = NRB_RED_THREADS / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) P.be_partials[v] = red[0];
        __syncthreads();  // red is reused by the next unit
    }
}

__global__ void k_b_be_derivatives(const BatchPair *__restrict__ pairs, const OptState *__restrict__ states,
                                   int npairs, BeBasis B) {
    __shared__ BatchList L;
    batch_list_build(states, npairs, 1u << PH_GRAD,
                     [&](int q, int& u, int& w) {
                         const BatchPair& b = pairs[q];
                         u = b.be_w > 0 ? (int)(3 * b.nnode) : 0;  // one element per (component, node)
                         w = 1;
                     }, L);
    batch_elements(L, [&](int p, long long e) {
        const BatchPair& P = pairs[p];
        const int k = (int)(e / P.nnode);
        const long long n = e - k * P.nnode;
        be_node_derivatives_k(P.cdim[0], P.cdim[1], P.cdim[2], P.grid_xyz, P.best, B, P.be_der, n, k);
    });
}

__global__ void k_b_be_accumulate(const BatchPair *__restrict__ pairs, const OptState *__restrict__ states,
                                  int npairs, BeBasis B) {
    __shared__ BatchList L;
    batch_list_build(states, npairs, 1u << PH_GRAD,
                     [&](int q, int& u, int& w) {
                         const BatchPair& b = pairs[q];
                         u = b.be_w > 0 ? (int)(3 * b.nnode) : 0;  // one element per (component, node)
                         w = 1;
                     }, L);
    batch_elements(L, [&](int p, long long e) {
        const BatchPair& P = pairs[p];
        const int k = (int)(e / P.nnode);
        const long long n = e - k * P.nnode;
        be_node_accumulate_k(P.cdim[0], P.cdim[1], P.cdim[2], P.be_der, B, P.be_ratio, P.grad, n, k);
    });
}

// x pass of the node convolution: work unit = one block of the plain k_conv_x
__global__ void __launch_bounds__(CONV_X_THREADS)
k_b_conv_x(const BatchPair *__restrict__ pairs, const OptState *__restrict__ states, int npairs) {
    extern __shared__ float rows[];
    __shared__ BatchList L;
    batch_list_build(states, npairs, 1u << PH_GRAD,
                     [&](int q, int& u, int& w) {
                         const BatchPair& b = pairs[q];
                         u = b.xblocks;
                         w = 1;
                     }, L);
    int k = 0;
    for (long long u = blockIdx.x; u < L.total; u += gridDim.x) {
        while (L.pref[k + 1] <= u) ++k;
        const BatchPair& P = pairs[L.pair[k]];
        conv_x_rows(P.rdim[0], P.rdim[1], P.rdim[2], P.vgrad, P.samples[0], P.ns[0], P.kernel[0], P.radius[0], P.conv1,
                    u - L.pref[k], rows);
        __syncthreads();  // rows are reused by the next unit
    }
}

// y pass ([3][nz][ny][nsx] -> [3][nz][nsy][nsx]) and z pass ([3][nz][nsy * nsx] ->
// [3][nsz][nsy * nsx]) of the node convolution, element-wise
__global__ void k_b_conv_y(const BatchPair *__restrict__ pairs, const OptState *__restrict__ states, int npairs) {
    __shared__ BatchList L;
    batch_list_build(states, npairs, 1u << PH_GRAD,
                     [&](int q, int& u, int& w) {
                         const BatchPair& b = pairs[q];
                         u = 3 * b.rdim[2] * b.ns[1] * b.ns[0];
                         w = 1;
                     }, L);
    batch_elements(L, [&](int p, long long i) {
        const BatchPair& P = pairs[p];
        conv_strided_at(P.rdim[2], P.rdim[1], P.ns[0], P.conv1, P.samples[1], P.ns[1], P.kernel[1], P.radius[1],
                        P.conv2, i);
    });
}

__global__ void k_b_conv_z(const BatchPair *__restrict__ pairs, const OptState *__restrict__ states, int npairs) {
    __shared__ BatchList L;
    batch_list_build(states, npairs, 1u << PH_GRAD,
                     [&](int q, int& u, int& w) {
                         const BatchPair& b = pairs[q];
                         u = 3 * b.ns[2] * b.ns[1] * b.ns[0];
                         w = 1;
                     }, L);
    batch_elements(L, [&](int p, long long i) {
        const BatchPair& P = pairs[p];
        conv_strided_at(1, P.rdim[2], P.ns[1] * P.ns[0], P.conv2, P.samples[2], P.ns[2], P.kernel[2], P.radius[2],
                        P.conv1, i);
    });
}

// node sampling, reorientation and weighting (overwrites the node gradient)
__global__ void k_b_nodes(const BatchPair *__restrict__ pairs, const OptState *__restrict__ states, int npairs) {
    __shared__ BatchList L;
    batch_list_build(states, npairs, 1u << PH_GRAD,
                     [&](int q, int& u, int& w) {
                         const BatchPair& b = pairs[q];
                         u = (int)b.nnode;
                         w = 1;
                     }, L);
    batch_elements(L, [&](int p, long long n) {
        const BatchPair& P = pairs[p];
        node_at(P.cdim[0], P.cdim[1], P.cdim[2], P.ns[0], P.ns[1], P.ns[2], P.conv1, P.tap_slot[0], P.tap_weight[0],
                P.tap_slot[1], P.tap_weight[1], P.tap_slot[2], P.tap_weight[2], P.flo_ijk, P.node_weight, P.grad, n);
    });
}

// ---------------------------------------------------------------------------------------------
// full-volume one-axis normalised convolution (value, density) pairs
// ---------------------------------------------------------------------------------------------
// din == nullptr: density = finite(vin) and NaN values count as 0 (first axis of a call).
__global__ void k_conv_axis(int nx, int ny, int nz, int axis, const float *__restrict__ vin,
                            const float *__restrict__ din, const float *__restrict__ K, int R,
                            float *__restrict__ vout, float *__restrict__ dout) {
    const long long nv = (long long)nx * ny * nz;
    const int n = axis == 0 ? nx : axis == 1 ? ny : nz;
    const long long stride = axis == 0 ? 1 : axis == 1 ? nx : (long long)nx * ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
         i += (long long)gridDim.x * blockDim.x) {
        const int p = axis == 0 ? (int)(i % nx) : axis == 1 ? (int)((i / nx) % ny) : (int)(i / ((long long)nx * ny));
        const long long base = i - (long long)p * stride;
        const int k0 = max(0, p - R), k1 = min(n - 1, p + R);
        float num = 0.f, den = 0.f;
        for (int k = k0; k <= k1; ++k) {
            const float w = K[k - p + R];
            float v = __ldg(&vin[base + k * stride]);
            float d;
            if (din) {
                d = __ldg(&din[base + k * stride]);
            } else {
                d = (v == v) ? 1.f : 0.f;
                if (v != v) v = 0.f;
            }
            num = fmaf(w, v, num);
            den = fmaf(w, d, den);
        }
        vout[i] = num;
        dout[i] = den;
    }
}

// value / density, NaN where the original value was NaN (_reg_tools.cpp:1100-1110)
__global__ void k_conv_normalise(long long nv, const float *orig, const float *__restrict__ v,
                                 const float *__restrict__ d, float *out) {  // out may alias orig
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
         i += (long long)gridDim.x * blockDim.x) {
        const float o = orig[i];
        out[i] = (o != o) ? o : v[i] / d[i];
    }
}

// float affine map in the reference's evaluation order, no contraction
__device__ __forceinline__ float affine_row_rn(const float *m, float x, float y, float z) {
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, m[0]), __fmul_rn(y, m[1])), __fmul_rn(z, m[2])), m[3]);
}

// Round<int> of reg-lib/cpu/Maths.hpp:83-85
__device__ __forceinline__ int round_ref(float x) { return (int)__fadd_rn(x, x >= 0.f ? 0.5f : -0.5f); }

// nearest-neighbour downsampling (reg_downsampleImage, reg-lib/cpu/_reg_tools.cpp:1343-1440):
// new voxel -> mm with the new qform, mm -> old voxel with the old one, rounded; NaN outside.
__global__ void k_downsample(int nx, int ny, int nz, int ox, int oy, int oz, Mat34 new_xyz,
                             Mat34 old_ijk, const float *__restrict__ in, float *__restrict__ out) {
    const long long nv = (long long)nx * ny * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
         i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long long)nx * ny));
        const float rx = affine_row_rn(new_xyz.m, (float)x, (float)y, (float)z);
        const float ry = affine_row_rn(new_xyz.m + 4, (float)x, (float)y, (float)z);
        const float rz = affine_row_rn(new_xyz.m + 8, (float)x, (float)y, (float)z);
        const float px = affine_row_rn(old_ijk.m, rx, ry, rz);
        const float py = affine_row_rn(old_ijk.m + 4, rx, ry, rz);
        const float pz = affine_row_rn(old_ijk.m + 8, rx, ry, rz);
        const int X = round_ref(px), Y = round_ref(py), Z = oz == 1 ? 0 : round_ref(pz);
        float v = __int_as_float(0x7fffffff);
        if (X > -1 && X < ox && Y > -1 && Y < oy && Z > -1 && Z < oz) v = in[((long long)Z * oy + Y) * ox + X];
        out[i] = v;
    }
}

// ---------------------------------------------------------------------------------------------
// reductions and element-wise updates
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(NRB_RED_THREADS)
k_minmax(long long n, const float *__restrict__ img, float *__restrict__ pmin, float *__restrict__ pmax) {
    __shared__ float smin[NRB_RED_THREADS], smax[NRB_RED_THREADS];
    float mn = FLT_MAX, mx = -FLT_MAX;
    for (long long i = blockIdx.x * (long long)NRB_RED_THREADS + threadIdx.x; i < n;
         i += (long long)gridDim.x * NRB_RED_THREADS) {
        const float v = img[i];
        if (v == v) {
            mn = fminf(mn, v);
            mx = fmaxf(mx, v);
        }
    }
    smin[threadIdx.x] = mn;
    smax[threadIdx.x] = mx;
    __syncthreads();
    for (int s = NRB_RED_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            smin[threadIdx.x] = fminf(smin[threadIdx.x], smin[threadIdx.x + s]);
            smax[threadIdx.x] = fmaxf(smax[threadIdx.x], smax[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        pmin[blockIdx.x] = smin[0];
        pmax[blockIdx.x] = smax[0];
    }
}

// reg_intensityRescale_core (reg-lib/cpu/_reg_tools.cpp:92-174): double-precision rescale of
// the finite values; every block combines the min/max partials itself.
__global__ void k_rescale(long long n, float *__restrict__ img, const float *__restrict__ pmin,
                          const float *__restrict__ pmax, int np, float new_min, float new_max) {
    __shared__ float mm[2];
    if (threadIdx.x == 0) {
        float mn = FLT_MAX, mx = -FLT_MAX;
        for (int i = 0; i < np; ++i) {
            mn = fminf(mn, pmin[i]);
            mx = fmaxf(mx, pmax[i]);
        }
        mm[0] = mn;
        mm[1] = mx;
    }
    __syncthreads();
    const double cur = (double)(mm[1] - mm[0]), nd = (double)(new_max - new_min), lo = (double)mm[0];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double v = (double)img[i];
        if (v == v) {
            v = (v - lo) / cur;
            v = v * nd + new_min;
        }
        img[i] = (float)v;
    }
}

// reg_getMaximalLength (reg-lib/cpu/_reg_tools.cpp:335-355): float lengths, max is exact in any
// order.
__global__ void __launch_bounds__(NRB_RED_THREADS)
k_maxlen(long long nnode, const float *__restrict__ g, float *__restrict__ pmax) {
    __shared__ float s[NRB_RED_THREADS];
    float mx = 0.f;
    for (long long i = blockIdx.x * (long long)NRB_RED_THREADS + threadIdx.x; i < nnode;
         i += (long long)gridDim.x * NRB_RED_THREADS) {
        const float x = g[i], y = g[nnode + i], z = g[2 * nnode + i];
        const float l = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
        mx = fmaxf(mx, l);
    }
    s[threadIdx.x] = mx;
    __syncthreads();
    for (int k = NRB_RED_THREADS / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) s[threadIdx.x] = fmaxf(s[threadIdx.x], s[threadIdx.x + k]);
        __syncthreads();
    }
    if (threadIdx.x == 0) pmax[blockIdx.x] = s[0];
}

__global__ void k_maxlen_finish(const float *__restrict__ pmax, int np, nrb_objective *__restrict__ obj,
                                double *__restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        float mx = 0.f;
        for (int i = 0; i < np; ++i) mx = fmaxf(mx, pmax[i]);
        if (obj) obj->max_grad_len = (double)mx;
        if (out) *out = (double)mx;
    }
}

// Compute::NormaliseGradient (reg-lib/Compute.cpp:148-176)
__global__ void k_normalise(long long n, float *__restrict__ g, const nrb_objective *__restrict__ obj,
                            double len) {
    const double l = len >= 0 ? len : obj->max_grad_len;
    if (l == 0) return;
    const double inv = 1.0 / l;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        g[i] = (float)((double)g[i] * inv);
}

// Compute::UpdateControlPointPosition (reg-lib/Compute.cpp:103-106)
__global__ void k_update(long long n, float *__restrict__ cur, const float *__restrict__ best,
                         const float *__restrict__ grad, float scale) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        cur[i] = __fadd_rn(best[i], __fmul_rn(scale, grad[i]));
}

// ConjugateGradient::UpdateGradientValues (reg-lib/Optimiser.cpp:231-317)
__global__ void k_cg_init(long long n, const float *__restrict__ g, float *__restrict__ g1, float *__restrict__ g2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float v = -g[i];
        g1[i] = v;
        g2[i] = v;
    }
}

__global__ void __launch_bounds__(NRB_RED_THREADS)
k_cg_dots(long long n, const float *__restrict__ g, const float *__restrict__ g1,
          const float *__restrict__ g2, double *__restrict__ partials) {
    __shared__ double red[NRB_RED_THREADS];
    double gg = 0, dgg = 0;
    for (long long i = blockIdx.x * (long long)NRB_RED_THREADS + threadIdx.x; i < n;
         i += (long long)gridDim.x * NRB_RED_THREADS) {
        gg += (double)__fmul_rn(g2[i], g1[i]);
        dgg += (double)__fmul_rn(__fadd_rn(g[i], g1[i]), g[i]);
    }
    const double a = block_sum_d(gg, red);
    __syncthreads();
    const double b = block_sum_d(dgg, red);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = a;
        partials[2 * blockIdx.x + 1] = b;
    }
}

// first_call (optional, device flag): when set, the first-call initialisation g1 = g2 = -g
// runs instead, so one captured launch serves both branches of UpdateGradientValues.
__global__ void k_cg_update(long long n, float *__restrict__ g, float *__restrict__ g1,
                            float *__restrict__ g2, const double *__restrict__ partials, int np,
                            const int *__restrict__ first_call) {
    if (first_call && *first_call) {
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
             i += (long long)gridDim.x * blockDim.x) {
            const float v = -g[i];
            g1[i] = v;
            g2[i] = v;
        }
        return;
    }
    // the partials are copied to shared memory by the whole block, then summed in index order by
    // two threads (gg and dgg side by side), instead of one thread's chain of global loads
    __shared__ double sp[2 * NRB_RED_BLOCKS];
    __shared__ double sgg, sdgg;
    for (int i = threadIdx.x; i < 2 * np; i += blockDim.x) sp[i] = partials[i];
    __syncthreads();
    if (threadIdx.x == 0 || threadIdx.x == 32) {
        const int q = threadIdx.x == 0 ? 0 : 1;
        double sum = 0;
        for (int i = 0; i < np; ++i) sum += sp[2 * i + q];
        if (q == 0) sgg = sum;
        else sdgg = sum;
    }
    __syncthreads();
    const double gm = sdgg / sgg;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float a1 = -g[i];
        const float a2 = (float)((double)a1 + gm * (double)g2[i]);
        g1[i] = a1;
        g2[i] = a2;
        g[i] = -a2;
    }
}

// ---------------------------------------------------------------------------------------------
// control-point grid construction and refinement
// ---------------------------------------------------------------------------------------------
// reg_createControlPointGrid's identity initialisation (reg_getDeformationFromDisplacement)
__global__ void k_grid_identity(int cx, int cy, int cz, Mat34 M, float *__restrict__ cpp) {
    const long long nc = (long long)cx * cy * cz;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nc;
         n += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(n % cx), y = (int)((n / cx) % cy), z = (int)(n / ((long long)cx * cy));
        for (int k = 0; k < 3; ++k) cpp[k * nc + n] = identity_pos(M, k, x, y, z);
    }
}

// reg_spline_refineControlPointGrid3D (reg-lib/cpu/_reg_localTrans.cpp:1809-2119): new node
// 2x-1 takes the (1,6,1)/8 mask around old node x, new node 2x the (1,1)/2 mask of x, x+1,
// per axis; old nodes outside the grid read as 0; new nodes past 2*old-2 are never written
// by the reference and stay 0.
__device__ __forceinline__ int refine_taps(int X, int oldn, int idx[3], int w[3]) {
    if ((X + 1) % 2 == 0) {
        const int x = (X + 1) / 2;
        if (x >= oldn) return 0;
        idx[0] = x - 1; idx[1] = x; idx[2] = x + 1;
        w[0] = 1; w[1] = 6; w[2] = 1;
        return 3;
    }
    const int x = X / 2;
    if (x >= oldn) return 0;
    idx[0] = x; idx[1] = x + 1;
    w[0] = 1; w[1] = 1;
    return 2;
}

__global__ void k_grid_refine(int ox, int oy, int oz, int nx, int ny, int nz, const float *__restrict__ old,
                              float *__restrict__ out) {
    const long long onc = (long long)ox * oy * oz, nnc = (long long)nx * ny * nz;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nnc;
         n += (long long)gridDim.x * blockDim.x) {
        const int X = (int)(n % nx), Y = (int)((n / nx) % ny), Z = (int)(n / ((long long)nx * ny));
        int ix[3], iy[3], iz[3], wx[3], wy[3], wz[3];
        const int ax = refine_taps(X, ox, ix, wx), ay = refine_taps(Y, oy, iy, wy), az = refine_taps(Z, oz, iz, wz);
        const float den = (float)((ax == 3 ? 8 : 2) * (ay == 3 ? 8 : 2) * (az == 3 ? 8 : 2));
        for (int k = 0; k < 3; ++k) {
            float v = 0.f;
            if (ax && ay && az) {
                // weight classes summed separately as the reference groups them
                float s1 = 0.f, s6 = 0.f, s36 = 0.f, s216 = 0.f;
                for (int c = 0; c < az; ++c)
                    for (int b = 0; b < ay; ++b)
                        for (int a = 0; a < ax; ++a) {
                            const int x = ix[a], y = iy[b], z = iz[c];
                            float val = 0.f;
                            if (x >= 0 && x < ox && y >= 0 && y < oy && z >= 0 && z < oz)
                                val = old[k * onc + ((long long)z * oy + y) * ox + x];
                            const int w = wx[a] * wy[b] * wz[c];
                            if (w == 1) s1 += val;
                            else if (w == 6) s6 += val;
                            else if (w == 36) s36 += val;
                            else s216 += val;
                        }
                v = (s1 + 6.f * s6 + 36.f * s36 + 216.f * s216) / den;
            }
            out[k * nnc + n] = v;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
static int grid_for(long long n, int threads, int max_blocks_per_sm = 16) {
    const long long want = (n + threads - 1) / threads;
    return (int)std::max<long long>(1, std::min<long long>(want, (long long)max_blocks_per_sm * sm_count()));
}

// Kernel width of reg_tools_kernelConvolution (_reg_tools.cpp:882-884): the spacing in mm over
// the voxel size, or |spacing| voxels when the spacing is negative; radius = int(2 * width).
// Refuses spacings and voxel sizes for which that is undefined (NaN, infinite, a voxel size that
// is not > 0 with a spacing in mm) and radii above 2^20 voxels.
static nrb_status cubic_extent(const char *who, float spacing_mm, float pixdim, double& temp, int& radius) {
    if (!std::isfinite(spacing_mm) || (spacing_mm > 0 && !(std::isfinite(pixdim) && pixdim > 0.f)))
        return fail(NRB_ERR_INVALID, std::string(who) + ": the spacing must be finite and, when given in mm, the "
                                                        "voxel size finite and > 0");
    temp = spacing_mm > 0 ? (double)(spacing_mm / pixdim) : std::fabs((double)spacing_mm);
    if (!(temp * 2.0 < (double)(1 << 20)))
        return fail(NRB_ERR_UNSUPPORTED, std::string(who) + ": kernel radius above 2^20 voxels");
    radius = (int)(temp * 2.0f);
    return NRB_OK;
}

// the 2 * radius + 1 cubic B-spline taps of reg_tools_kernelConvolution (_reg_tools.cpp:893-904)
static void cubic_taps(double temp, int radius, float *out) {
    for (int i = -radius; i <= radius; ++i) {
        const double rel = std::fabs(i / temp);
        float v;
        if (rel < 1.0) v = (float)(2.0 / 3.0 - rel * rel + 0.5 * rel * rel * rel);
        else if (rel < 2.0) v = (float)(-(rel - 2.0) * (rel - 2.0) * (rel - 2.0) / 6.0);
        else v = 0.f;
        out[i + radius] = v;
    }
}

// cubic B-spline convolution kernel of a geometry the workspace has already validated
static std::vector<float> cubic_kernel(float spacing_mm, float pixdim, int& radius) {
    const double temp = spacing_mm > 0 ? (double)(spacing_mm / pixdim) : std::fabs((double)spacing_mm);
    radius = (int)(temp * 2.0f);
    std::vector<float> k(2 * radius + 1);
    cubic_taps(temp, radius, k.data());
    return k;
}

// ref_ijk * cpp_xyz (mat44 product, entries rounded to float): the grid's node -> reference
// voxel map; aligned when its 3x3 part is diagonal (to 1e-6 relative), as every grid built by
// reg_createControlPointGrid / refinement is for its reference
static void node_to_voxel(const nrb_geometry *g, double T[3][4]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0;
            for (int k = 0; k < 4; ++k) s += (double)g->ref_ijk[4 * i + k] * (double)g->cpp_xyz[4 * k + j];
            T[i][j] = (float)s;
        }
}
static bool grid_aligned(const nrb_geometry *g) {
    double T[3][4];
    node_to_voxel(g, T);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (i != j && std::fabs(T[i][j]) > 1e-6 * std::fabs(T[i][i])) return false;
    return true;
}

nrb_status validate_geometry(const nrb_geometry *g) {
    // voxel and node indices are 32-bit in the kernels
    if (nvox(g->ref_dim) >= (1LL << 31) / 3 || nvox(g->flo_dim) >= (1LL << 31) || nvox(g->cpp_dim) >= (1LL << 31) / 3)
        return fail(NRB_ERR_UNSUPPORTED, "geometry: volume too large for 32-bit indexing");
    for (int d = 0; d < 3; ++d) {
        if (g->ref_dim[d] <= 0 || g->flo_dim[d] <= 0 || g->cpp_dim[d] <= 0)
            return fail(NRB_ERR_INVALID, "geometry: non-positive dimension");
        if (!(g->ref_pixdim[d] > 0) || !(g->cpp_pixdim[d] > 0))
            return fail(NRB_ERR_INVALID, "geometry: non-positive voxel size");
        if (g->ref_dim[d] > 2048) return fail(NRB_ERR_UNSUPPORTED, "geometry: dimension above 2048");
        const float gs = g->cpp_pixdim[d] / g->ref_pixdim[d];
        if (gs < 1.f) return fail(NRB_ERR_UNSUPPORTED, "geometry: control spacing below one voxel");
        const int last = (int)((float)(g->ref_dim[d] - 1) / gs);
        // the aligned passes address nodes from voxel indices; an unaligned grid is sampled
        // through its full matrix (0 outside), so only an aligned grid must cover the reference
        if (last + 3 >= g->cpp_dim[d] && grid_aligned(g))
            return fail(NRB_ERR_UNSUPPORTED, "geometry: control-point grid does not cover the reference");
    }
    return NRB_OK;
}

static int tile_span(int n, int tile, float gs) {
    int span = 0;
    for (int v0 = 0; v0 < n; v0 += tile) {
        const int v1 = std::min(v0 + tile - 1, n - 1);
        span = std::max(span, (int)((float)v1 / gs) + 4 - (int)((float)v0 / gs));
    }
    return span;
}

// Node -> reference voxel sampling per axis (reg_voxelCentricToNodeCentric,
// _reg_localTrans.cpp:1572-1631): requires ref_ijk * cpp_xyz to be axis-aligned, which holds
// for every grid built by reg_createControlPointGrid / refinement.
static nrb_status make_sampling(const nrb_geometry *g, AxisSampling ax[3]) {
    double T[3][4];
    node_to_voxel(g, T);  // mat44 operator* rounds each entry to float
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (i != j && std::fabs(T[i][j]) > 1e-6 * std::fabs(T[i][i]))
                return fail(NRB_ERR_UNSUPPORTED, "voxel->node: grid not axis-aligned with the reference");
    for (int d = 0; d < 3; ++d) {
        AxisSampling& a = ax[d];
        const int n = g->ref_dim[d], cn = g->cpp_dim[d];
        std::vector<int> pre(cn);
        std::vector<float> w1(cn);
        std::vector<int> used;
        for (int i = 0; i < cn; ++i) {
            const float v = (float)(T[d][d] * (double)i + T[d][3]);
            pre[i] = (int)std::floor(v);
            w1[i] = v - (float)pre[i];
            if (pre[i] >= 0 && pre[i] < n) used.push_back(pre[i]);
            if (w1[i] != 0.f && pre[i] + 1 >= 0 && pre[i] + 1 < n) used.push_back(pre[i] + 1);
        }
        std::sort(used.begin(), used.end());
        used.erase(std::unique(used.begin(), used.end()), used.end());
        if (used.empty()) used.push_back(0);  // keep buffers non-empty; no node reads it
        a.samples = used;
        a.nsamples = (int)used.size();
        a.tap_slot.assign(2 * cn, -1);
        a.tap_weight.assign(2 * cn, 0.f);
        for (int i = 0; i < cn; ++i) {
            const float w0 = 1.f - w1[i];
            if (pre[i] >= 0 && pre[i] < n) {
                a.tap_slot[2 * i] = (int)(std::lower_bound(used.begin(), used.end(), pre[i]) - used.begin());
                a.tap_weight[2 * i] = w0;
            }
            if (w1[i] != 0.f && pre[i] + 1 >= 0 && pre[i] + 1 < n) {
                a.tap_slot[2 * i + 1] = (int)(std::lower_bound(used.begin(), used.end(), pre[i] + 1) - used.begin());
                a.tap_weight[2 * i + 1] = w1[i];
            }
        }
        a.kernel = cubic_kernel(g->cpp_pixdim[d], g->ref_pixdim[d], a.radius);
    }
    return NRB_OK;
}

// The source vectors live as long as the workspace, so the stream-ordered copy may finish later.
template <typename T>
static nrb_status upload(T *&dst, const std::vector<T>& src, size_t& bytes, cudaStream_t st) {
    NRB_CUDA(dev_alloc(&dst, std::max<size_t>(1, src.size()) * sizeof(T), st));
    if (!src.empty()) {
        if (st) NRB_CUDA(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, st));
        else NRB_CUDA(cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    }
    bytes += src.size() * sizeof(T);
    return NRB_OK;
}

// Items of the voxel walk. The persistent grid holds slots_for(shared bytes) co-resident blocks
// and every block walks ceil(items / slots) items, so the z-chunk count is chosen to minimise a
// block's walk: rounds x (slices per chunk + the item's fixed cost, `overhead` slices: staging,
// the x rows, the column set-up), over chunk counts that keep chunks at least `min_chunk`
// slices long (the staged control points are reused along z). Small volumes, whose few long
// items would leave most blocks idle, get shorter chunks spread over more blocks.
WalkPlan plan_walk(const nrb_geometry *g, int ty, long long (*slots_for)(size_t smem), size_t extra_smem,
                   int min_chunk, int overhead) {
    WalkPlan p;
    p.ty = ty;
    const int nx = g->ref_dim[0], ny = g->ref_dim[1], nz = g->ref_dim[2];
    const float gs[3] = { g->cpp_pixdim[0] / g->ref_pixdim[0], g->cpp_pixdim[1] / g->ref_pixdim[1],
                          g->cpp_pixdim[2] / g->ref_pixdim[2] };
    p.tiles_x = (nx + COL_X - 1) / COL_X;
    p.tiles_y = (ny + ty - 1) / ty;
    const long long xy = (long long)p.tiles_x * p.tiles_y;
    p.sa = tile_span(nx, COL_X, gs[0]);
    p.sb = tile_span(ny, ty, gs[1]);
    long long best_cost = LLONG_MAX;
    WalkPlan best = p;
    for (int c = 1; c <= std::max(1, nz / min_chunk); ++c) {
        WalkPlan q = p;
        q.zchunk = (nz + c - 1) / c;
        q.nchunks = (nz + q.zchunk - 1) / q.zchunk;
        q.nitems = (int)(xy * q.nchunks);
        q.sc = tile_span(nz, q.zchunk, gs[2]);
        q.cp_floats = 3 * q.sa * q.sb * q.sc;
        const long long slots = std::max(1LL, slots_for(walk_smem_bytes(q) + extra_smem));
        const long long rounds = (q.nitems + slots - 1) / slots;
        const long long cost = rounds * (q.zchunk + overhead);
        if (cost < best_cost) {
            best_cost = cost;
            best = q;
        }
    }
    return best;
}

std::vector<WalkPlan> plan_walk_candidates(const nrb_geometry *g, int ty, long long (*slots_for)(size_t smem),
                                           size_t extra_smem, int min_chunk, int overhead, int count) {
    const int nx = g->ref_dim[0], ny = g->ref_dim[1], nz = g->ref_dim[2];
    const float gs[3] = { g->cpp_pixdim[0] / g->ref_pixdim[0], g->cpp_pixdim[1] / g->ref_pixdim[1],
                          g->cpp_pixdim[2] / g->ref_pixdim[2] };
    WalkPlan p;
    p.ty = ty;
    p.tiles_x = (nx + COL_X - 1) / COL_X;
    p.tiles_y = (ny + ty - 1) / ty;
    p.sa = tile_span(nx, COL_X, gs[0]);
    p.sb = tile_span(ny, ty, gs[1]);
    const long long xy = (long long)p.tiles_x * p.tiles_y;
    std::vector<std::pair<long long, WalkPlan>> all;
    int last_chunk = -1;
    for (int c = 1; c <= std::max(1, nz / min_chunk); ++c) {
        WalkPlan q = p;
        q.zchunk = (nz + c - 1) / c;
        if (q.zchunk == last_chunk) continue;
        last_chunk = q.zchunk;
        q.nchunks = (nz + q.zchunk - 1) / q.zchunk;
        q.nitems = (int)(xy * q.nchunks);
        q.sc = tile_span(nz, q.zchunk, gs[2]);
        q.cp_floats = 3 * q.sa * q.sb * q.sc;
        const long long slots = std::max(1LL, slots_for(walk_smem_bytes(q) + extra_smem));
        const long long rounds = (q.nitems + slots - 1) / slots;
        all.emplace_back(rounds * (q.zchunk + overhead), q);
    }
    std::stable_sort(all.begin(), all.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    std::vector<WalkPlan> out;
    for (size_t i = 0; i < all.size() && (int)out.size() < count; ++i) out.push_back(all[i].second);
    return out;
}

nrb_status workspace_init(nrb_workspace *ws, const nrb_geometry *g) {
    ws->g = *g;
    // shared memory beyond the walk: the 64-bin joint histogram / FP32 log table (the plan is
    // made before the bin count is known; other bin counts shift occupancy little)
    ws->walk_obj = plan_walk(g, TY_OBJECTIVE, objective_slots, OBJ_PLAN_EXTRA, 4, 6);
    ws->walk_grad = plan_walk(g, TY_GRADIENT, gradient_slots, GRAD_PLAN_EXTRA, 4, 4);
    return NRB_OK;
}

static nrb_status workspace_alloc(nrb_workspace *ws) {
    const nrb_geometry *g = &ws->g;
    NRB_CUDA(cudaGetDevice(&ws->device));
    size_t bytes = 0;
    if (!grid_aligned(g)) {
        // the whole-volume convolution and per-node sampling replace the separable passes
        ws->general = true;
        const size_t vb = (size_t)3 * nvox(g->ref_dim) * 4;
        if (dev_alloc(&ws->general_vox, vb, ws->st) != cudaSuccess) {
            cudaGetLastError();
            return fail(NRB_ERR_OOM, "workspace allocation failed");
        }
        bytes += vb;
        for (int d = 0; d < 3; ++d) {
            ws->ax[d] = AxisSampling{};
            ws->ax[d].samples.assign(1, 0);
            ws->ax[d].nsamples = 1;
        }
    } else {
        NRB_TRY(make_sampling(g, ws->ax));
    }
    for (int d = 0; d < 3; ++d) {
        NRB_TRY(upload(ws->d_samples[d], ws->ax[d].samples, bytes, ws->st));
        NRB_TRY(upload(ws->d_tap_slot[d], ws->ax[d].tap_slot, bytes, ws->st));
        NRB_TRY(upload(ws->d_tap_weight[d], ws->ax[d].tap_weight, bytes, ws->st));
        NRB_TRY(upload(ws->d_kernel[d], ws->ax[d].kernel, bytes, ws->st));
    }
    const long long nx = g->ref_dim[0], ny = g->ref_dim[1], nz = g->ref_dim[2];
    const long long c1 = 3LL * nz * ny * ws->ax[0].nsamples;
    const long long c2 = 3LL * nz * ws->ax[1].nsamples * ws->ax[0].nsamples;
    const long long c3 = 3LL * ws->ax[2].nsamples * ws->ax[1].nsamples * ws->ax[0].nsamples;
    (void)nx;
    const long long nc = nvox(g->cpp_dim);
    const size_t sz1 = (size_t)std::max(c1, c3) * 4, sz2 = (size_t)c2 * 4;
    cudaStream_t st = ws->st;
    if (dev_alloc(&ws->conv1, sz1, st) != cudaSuccess || dev_alloc(&ws->conv2, sz2, st) != cudaSuccess ||
        dev_alloc(&ws->be_deriv, (size_t)18 * nc * 4, st) != cudaSuccess ||
        dev_alloc(&ws->red, 2 * NRB_RED_BLOCKS * sizeof(double), st) != cudaSuccess ||
        dev_alloc(&ws->be_partials, NRB_RED_BLOCKS * sizeof(double), st) != cudaSuccess ||
        dev_alloc(&ws->fred, 2 * NRB_RED_BLOCKS * sizeof(float), st) != cudaSuccess) {
        cudaGetLastError();
        return fail(NRB_ERR_OOM, "workspace allocation failed");
    }
    bytes += sz1 + sz2 + (size_t)18 * nc * 4 + 3 * NRB_RED_BLOCKS * sizeof(double) + 2 * NRB_RED_BLOCKS * 4;
    ws->bytes = bytes;
    NRB_CUDA(cudaStreamCreateWithFlags(&ws->side, cudaStreamNonBlocking));
    NRB_CUDA(cudaEventCreateWithFlags(&ws->ev_fork, cudaEventDisableTiming));
    NRB_CUDA(cudaEventCreateWithFlags(&ws->ev_join, cudaEventDisableTiming));
    return NRB_OK;
}

nrb_status fork_side(nrb_workspace *ws, cudaStream_t st) {
    NRB_CUDA(cudaEventRecord(ws->ev_fork, st));
    NRB_CUDA(cudaStreamWaitEvent(ws->side, ws->ev_fork, 0));
    return NRB_OK;
}

nrb_status join_side(nrb_workspace *ws, cudaStream_t st) {
    NRB_CUDA(cudaEventRecord(ws->ev_join, ws->side));
    NRB_CUDA(cudaStreamWaitEvent(st, ws->ev_join, 0));
    return NRB_OK;
}

void workspace_free(nrb_workspace *ws) {
    cudaStream_t st = ws->st;
    for (int d = 0; d < 3; ++d) {
        dev_free(ws->d_samples[d], st);
        dev_free(ws->d_tap_slot[d], st);
        dev_free(ws->d_tap_weight[d], st);
        dev_free(ws->d_kernel[d], st);
    }
    dev_free(ws->conv1, st);
    dev_free(ws->conv2, st);
    dev_free(ws->general_vox, st);
    dev_free(ws->be_deriv, st);
    dev_free(ws->red, st);
    dev_free(ws->be_partials, st);
    dev_free(ws->fred, st);
    // the side stream's work is ordered before st's last join; its frees above are on st
    if (ws->ev_fork) cudaEventDestroy(ws->ev_fork);
    if (ws->ev_join) cudaEventDestroy(ws->ev_join);
    if (ws->side) cudaStreamDestroy(ws->side);
}

static int be_grid(const nrb_geometry *g) {
    const long long ni = (long long)std::max(0, g->cpp_dim[0] - 2) * std::max(0, g->cpp_dim[1] - 2) *
                         std::max(0, g->cpp_dim[2] - 2);
    return (int)std::max<long long>(1, std::min<long long>((ni + NRB_RED_THREADS - 1) / NRB_RED_THREADS, NRB_RED_BLOCKS));
}

nrb_status launch_be_value(nrb_workspace *ws, const nrb_geometry *g, const float *cpp, cudaStream_t st,
                           const float *grad, const OptState *step) {
    const int grid = be_grid(g);
    KernelTimer timer(TK_BE_VALUE, 12.0 * (double)nvox(g->cpp_dim), st);
    k_be_value<<<grid, 3 * NRB_RED_THREADS, 0, st>>>(g->cpp_dim[0], g->cpp_dim[1], g->cpp_dim[2], cpp, be_basis(),
                                                  ws->be_partials, grad, step);
    NRB_LAUNCHED("k_be_value");
    return NRB_OK;
}

int be_partial_count(const nrb_geometry *g) { return be_grid(g); }

nrb_status voxel_to_node_general(const float *vox, const nrb_geometry *g, float weight, float *node,
                                 cudaStream_t st);

nrb_status launch_convolve_to_nodes(nrb_workspace *ws, const nrb_geometry *g, const float *vgrad,
                                    float weight, float *node, cudaStream_t st) {
    if (ws->general) {
        // Compute::ConvolveVoxelBasedMeasureGradient (reg-lib/Compute.cpp:230-281) as written:
        // the whole gradient convolved along the image axes with the grid spacings, then every
        // node sampled through the full node -> voxel matrix
        KernelTimer timer(TK_CONV, 0.0, st);
        const long long nv = nvox(g->ref_dim);
        NRB_CUDA(cudaMemcpyAsync(ws->general_vox, vgrad, 3 * nv * sizeof(float), cudaMemcpyDeviceToDevice, st));
        for (int axis = 0; axis < 3; ++axis)
            NRB_TRY(nrb_kernel_convolution_cubic(ws->general_vox, 3, g->ref_dim, g->ref_pixdim, g->cpp_pixdim[axis],
                                                 axis, st));
        return voxel_to_node_general(ws->general_vox, g, weight, node, st);
    }
    const int nx = g->ref_dim[0], ny = g->ref_dim[1], nz = g->ref_dim[2];
    const int nsx = ws->ax[0].nsamples, nsy = ws->ax[1].nsamples, nsz = ws->ax[2].nsamples;
    // compulsory traffic of the whole voxel->node step: the voxel gradient once, the nodes once
    KernelTimer timer(TK_CONV, 12.0 * (double)nx * ny * nz + 12.0 * (double)nvox(g->cpp_dim), st);
    // x pass: one block per row
    // rows | kernel taps | per-sample weight sums (nx <= 2048: <= 205 KB)
    const size_t smem = ((size_t)3 * CONV_X_ROWS * nx + 2 * ws->ax[0].radius + 1 + nsx) * 4;
    if (smem > 227 * 1024) return fail(NRB_ERR_UNSUPPORTED, "convolution: rows and kernel exceed shared memory");
    if (smem > 48 * 1024) NRB_CUDA(cudaFuncSetAttribute(k_conv_x, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int xblocks = (int)(((long long)ny * nz + CONV_X_ROWS - 1) / CONV_X_ROWS);
    k_conv_x<<<xblocks, CONV_X_THREADS, smem, st>>>(nx, ny, nz, vgrad, ws->d_samples[0], nsx, ws->d_kernel[0],
                                         ws->ax[0].radius, ws->conv1);
    NRB_LAUNCHED("k_conv_x");
    // y pass: [3][nz][ny][nsx] -> [3][nz][nsy][nsx]
    long long t2 = 3LL * nz * nsy * nsx;
    k_conv_strided<<<grid_for(t2, 256), 256, 0, st>>>(nz, ny, nsx, ws->conv1, ws->d_samples[1], nsy,
                                                      ws->d_kernel[1], ws->ax[1].radius, ws->conv2);
    NRB_LAUNCHED("k_conv_strided(y)");
    // z pass: [3][1][nz][nsy*nsx] -> [3][nsz][nsy*nsx] (reuses conv1)
    long long t3 = 3LL * nsz * nsy * nsx;
    k_conv_strided<<<grid_for(t3, 256), 256, 0, st>>>(1, nz, nsy * nsx, ws->conv2, ws->d_samples[2], nsz,
                                                      ws->d_kernel[2], ws->ax[2].radius, ws->conv1);
    NRB_LAUNCHED("k_conv_strided(z)");
    // node sampling, reorientation (floating ijk) and weighting
    float w = weight;
    for (int i = 0; i < 3; ++i) w *= g->cpp_pixdim[i] / g->ref_pixdim[i];
    const long long nc = nvox(g->cpp_dim);
    k_nodes<<<grid_for(nc, 256), 256, 0, st>>>(g->cpp_dim[0], g->cpp_dim[1], g->cpp_dim[2], nsx, nsy, nsz, ws->conv1,
                                               ws->d_tap_slot[0], ws->d_tap_weight[0], ws->d_tap_slot[1],
                                               ws->d_tap_weight[1], ws->d_tap_slot[2], ws->d_tap_weight[2],
                                               to_mat34(g->flo_ijk), w, node);
    NRB_LAUNCHED("k_nodes");
    return NRB_OK;
}

}  // namespace nrb

using namespace nrb;

// ---------------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------------
nrb_status nrb::workspace_create_on(const nrb_geometry *g, cudaStream_t st, nrb_workspace **out) {
    if (!g || !out) return fail(NRB_ERR_INVALID, "nrb_workspace_create: null pointer");
    NRB_TRY(validate_geometry(g));
    nrb_workspace *ws = new nrb_workspace();
    ws->st = st;
    nrb_status s = workspace_init(ws, g);
    if (s == NRB_OK) s = workspace_alloc(ws);
    if (s != NRB_OK) {
        workspace_free(ws);
        delete ws;
        return s;
    }
    *out = ws;
    return NRB_OK;
}

extern "C" nrb_status nrb_workspace_create(const nrb_geometry *g, nrb_workspace **out) {
    if (!g || !out) return fail(NRB_ERR_INVALID, "nrb_workspace_create: null pointer");
    NRB_TRY(validate_geometry(g));
    nrb_workspace *ws = new nrb_workspace();
    nrb_status s = workspace_init(ws, g);
    if (s == NRB_OK) s = workspace_alloc(ws);
    if (s != NRB_OK) {
        workspace_free(ws);
        delete ws;
        return s;
    }
    *out = ws;
    return NRB_OK;
}

extern "C" void nrb_workspace_destroy(nrb_workspace *ws) {
    if (!ws) return;
    workspace_free(ws);
    delete ws;
}

extern "C" nrb_status nrb_convolve_voxel_based_gradient(nrb_workspace *ws, const nrb_geometry *g,
                                                        const float *vgrad, float weight,
                                                        float *node_grad, void *stream) {
    if (!ws || !g || !vgrad || !node_grad) return fail(NRB_ERR_INVALID, "nrb_convolve_voxel_based_gradient: null pointer");
    return launch_convolve_to_nodes(ws, g, vgrad, weight, node_grad, as_stream(stream));
}

extern "C" nrb_status nrb_kernel_convolution_cubic(float *img, int nvol, const int32_t dim[3],
                                                   const float pixdim[3], float spacing_mm, int axis,
                                                   void *stream) {
    if (!img || !dim || !pixdim || nvol <= 0 || axis < 0 || axis > 2)
        return fail(NRB_ERR_INVALID, "nrb_kernel_convolution_cubic: bad argument");
    cudaStream_t st = as_stream(stream);
    double temp = 0;
    int radius = 0;
    NRB_TRY(cubic_extent("nrb_kernel_convolution_cubic", spacing_mm, pixdim[axis], temp, radius));
    if (radius <= 0 || dim[axis] <= 1) return NRB_OK;  // the reference leaves the image as is
    std::vector<float> k(2 * radius + 1);
    cubic_taps(temp, radius, k.data());
    const long long nv = (long long)dim[0] * dim[1] * dim[2];
    float *dk = nullptr, *tv = nullptr, *td = nullptr;
    NRB_CUDA(tmp_alloc(&dk, k.size() * 4, st));
    NRB_CUDA(tmp_alloc(&tv, nv * 4, st));
    NRB_CUDA(tmp_alloc(&td, nv * 4, st));
    NRB_CUDA(cudaMemcpyAsync(dk, k.data(), k.size() * 4, cudaMemcpyHostToDevice, st));
    for (int t = 0; t < nvol; ++t) {
        float *v = img + t * nv;
        k_conv_axis<<<grid_for(nv, 256), 256, 0, st>>>(dim[0], dim[1], dim[2], axis, v, nullptr, dk, radius, tv, td);
        NRB_LAUNCHED("k_conv_axis");
        k_conv_normalise<<<grid_for(nv, 256), 256, 0, st>>>(nv, v, tv, td, v);
        NRB_LAUNCHED("k_conv_normalise");
    }
    NRB_CUDA(cudaFreeAsync(dk, st));
    NRB_CUDA(cudaFreeAsync(tv, st));
    NRB_CUDA(cudaFreeAsync(td, st));
    return NRB_OK;
}

// ---------------------------------------------------------------------------------------------
// The same convolution with its scratch in a fixed, module-level device array.
//
// Some callers cannot allocate device memory at the moment they need this convolution: code
// that is recording a CUDA stream capture (an allocation there either fails or becomes part of
// the graph), code running under a hard per-process memory cap that is already spent, or code
// that hands out device memory from its own pool and forbids the library from touching the
// driver's allocator. For them the scratch (the kernel taps and the value/density pair of one
// volume) lives in `g_static_scratch`, which the module reserves when it is loaded.
//
// Layout: [taps: NRB_STATIC_CONV_MAX_TAPS floats, padded to 256 B][value: max voxels floats]
// [density: max voxels floats]. Nothing in it has to start at zero: every call writes the taps
// and then both temporaries of a volume in full before it reads them.
//
// There is one scratch per device and no lock: two calls whose kernels can overlap on the same
// device (different streams without ordering, or different host threads) race on it.
// ---------------------------------------------------------------------------------------------
namespace {

constexpr size_t kStaticTapBytes = 256 * ((NRB_STATIC_CONV_MAX_TAPS * sizeof(float) + 255) / 256);
constexpr size_t kStaticScratchBytes = kStaticTapBytes + 2 * sizeof(float) * (size_t)NRB_STATIC_CONV_MAX_VOXELS;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// the taps travel as a kernel argument, so no host-to-device copy is needed for them
struct StaticTaps {
    float k[NRB_STATIC_CONV_MAX_TAPS];
};

__global__ void k_static_taps(const __grid_constant__ StaticTaps t, int n, float *__restrict__ dst) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = t.k[i];
}

// Address of this device's scratch. cudaGetSymbolAddress runs once per device, with that device
// current (the caller's current device); later calls read the cached pointer.
constexpr int kMaxDevices = 64;
std::mutex g_static_mutex;
unsigned char *g_static_addr[kMaxDevices] = {};

nrb_status static_scratch(unsigned char **out) {
    int dev = 0;
    NRB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(NRB_ERR_UNSUPPORTED, "static scratch: device index above 63");
    std::lock_guard<std::mutex> lock(g_static_mutex);
    if (!g_static_addr[dev]) {
        void *p = nullptr;
        NRB_CUDA(cudaGetSymbolAddress(&p, g_static_scratch));
        g_static_addr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_static_addr[dev];
    return NRB_OK;
}

}  // namespace

extern "C" nrb_status nrb_kernel_convolution_cubic_static(float *img, int nvol, const int32_t dim[3],
                                                          const float pixdim[3], float spacing_mm, int axis,
                                                          void *stream) {
    if (!img || !dim || !pixdim || nvol <= 0 || axis < 0 || axis > 2 || dim[0] <= 0 || dim[1] <= 0 || dim[2] <= 0)
        return fail(NRB_ERR_INVALID, "nrb_kernel_convolution_cubic_static: bad argument");
    const long long nv = (long long)dim[0] * dim[1] * dim[2];
    if (nv > NRB_STATIC_CONV_MAX_VOXELS)
        return fail(NRB_ERR_UNSUPPORTED, "nrb_kernel_convolution_cubic_static: volume has more voxels than the "
                                         "static scratch holds (NRB_STATIC_CONV_MAX_VOXELS = 2097152)");
    double temp = 0;
    int radius = 0;
    NRB_TRY(cubic_extent("nrb_kernel_convolution_cubic_static", spacing_mm, pixdim[axis], temp, radius));
    // the same early return as the allocating entry point, before the size limit on the taps
    if (radius <= 0 || dim[axis] <= 1) return NRB_OK;  // the reference leaves the image as is
    if (2 * radius + 1 > NRB_STATIC_CONV_MAX_TAPS)
        return fail(NRB_ERR_UNSUPPORTED, "nrb_kernel_convolution_cubic_static: kernel wider than the static "
                                         "scratch holds (NRB_STATIC_CONV_MAX_TAPS = 511 taps)");
    StaticTaps taps;
    cubic_taps(temp, radius, taps.k);
    unsigned char *base = nullptr;
    NRB_TRY(static_scratch(&base));
    float *dk = reinterpret_cast<float *>(base);
    float *tv = reinterpret_cast<float *>(base + kStaticTapBytes);
    float *td = tv + NRB_STATIC_CONV_MAX_VOXELS;
    cudaStream_t st = as_stream(stream);
    k_static_taps<<<1, 256, 0, st>>>(taps, 2 * radius + 1, dk);
    NRB_LAUNCHED("k_static_taps");
    for (int t = 0; t < nvol; ++t) {
        float *v = img + t * nv;
        k_conv_axis<<<grid_for(nv, 256), 256, 0, st>>>(dim[0], dim[1], dim[2], axis, v, nullptr, dk, radius, tv, td);
        NRB_LAUNCHED("k_conv_axis");
        k_conv_normalise<<<grid_for(nv, 256), 256, 0, st>>>(nv, v, tv, td, v);
        NRB_LAUNCHED("k_conv_normalise");
    }
    return NRB_OK;
}

extern "C" nrb_status nrb_approx_bending_energy(nrb_workspace *ws, const nrb_geometry *g, const float *cpp,
                                                nrb_objective *obj, double *be_host, void *stream) {
    if (!ws || !g || !cpp) return fail(NRB_ERR_INVALID, "nrb_approx_bending_energy: null pointer");
    cudaStream_t st = as_stream(stream);
    NRB_TRY(launch_be_value(ws, g, cpp, st));
    nrb_objective *o = obj;
    nrb_objective *tmp = nullptr;
    if (!o) {
        NRB_CUDA(tmp_alloc(&tmp, sizeof(nrb_objective), st));
        o = tmp;
    }
    k_be_sum<<<1, NRB_RED_THREADS, 0, st>>>(ws->be_partials, be_grid(g), 3.0 * (double)nvox(g->cpp_dim), o);
    NRB_LAUNCHED("k_be_sum");
    if (be_host) {
        NRB_CUDA(cudaMemcpyAsync(be_host, &o->be, sizeof(double), cudaMemcpyDeviceToHost, st));
        NRB_CUDA(cudaStreamSynchronize(st));
    }
    if (tmp) NRB_CUDA(cudaFreeAsync(tmp, st));
    return NRB_OK;
}

namespace nrb {
// reg_spline_approxBendingEnergyGradient3D, first half: the 18 second-derivative values of
// every node (grid read, derivatives written)
nrb_status launch_be_derivatives(nrb_workspace *ws, const nrb_geometry *g, const float *cpp, cudaStream_t st) {
    const long long nc = nvox(g->cpp_dim);
    KernelTimer timer(TK_BE_GRADIENT, (12.0 + 72.0) * (double)nc, st);
    k_be_derivatives<<<dim3(grid_for(nc, 128), 3), 128, 0, st>>>(g->cpp_dim[0], g->cpp_dim[1], g->cpp_dim[2],
                                                        to_mat34(g->cpp_xyz), cpp, be_basis(), ws->be_deriv);
    NRB_LAUNCHED("k_be_derivatives");
    return NRB_OK;
}

// second half: the adjoint stencil, node_grad += weight / #nodes * sum (derivatives read,
// gradient read-modify-write)
nrb_status launch_be_accumulate(nrb_workspace *ws, const nrb_geometry *g, float weight, float *node_grad,
                                cudaStream_t st) {
    const long long nc = nvox(g->cpp_dim);
    KernelTimer timer(TK_BE_GRADIENT, (72.0 + 24.0) * (double)nc, st);
    const float ratio = weight / (float)nc;
    k_be_accumulate<<<dim3(grid_for(nc, 128), 3), 128, 0, st>>>(g->cpp_dim[0], g->cpp_dim[1], g->cpp_dim[2], ws->be_deriv,
                                                       be_basis(), ratio, node_grad);
    NRB_LAUNCHED("k_be_accumulate");
    return NRB_OK;
}

// ---- batched levels -------------------------------------------------------------------------
// A pair's node-stage description: its workspace's convolution sampling and bending-energy
// buffers, as launch_convolve_to_nodes / launch_be_* use them for its geometry.
nrb_status batch_node_stage(const nrb_workspace *ws, const nrb_geometry *g, float sim_weight, float be_weight,
                            BatchPair& b) {
    if (ws->general) return fail(NRB_ERR_UNSUPPORTED, "batched level: the grid must be aligned with the reference");
    for (int i = 0; i < 3; ++i) {
        b.rdim[i] = g->ref_dim[i];
        b.cdim[i] = g->cpp_dim[i];
        b.ns[i] = ws->ax[i].nsamples;
        b.radius[i] = ws->ax[i].radius;
        b.samples[i] = ws->d_samples[i];
        b.tap_slot[i] = ws->d_tap_slot[i];
        b.tap_weight[i] = ws->d_tap_weight[i];
        b.kernel[i] = ws->d_kernel[i];
    }
    b.nnode = nvox(g->cpp_dim);
    b.conv1 = ws->conv1;
    b.conv2 = ws->conv2;
    float w = sim_weight;
    for (int i = 0; i < 3; ++i) w *= g->cpp_pixdim[i] / g->ref_pixdim[i];
    b.node_weight = w;
    b.flo_ijk = to_mat34(g->flo_ijk);
    b.grid_xyz = to_mat34(g->cpp_xyz);
    b.be_partials = ws->be_partials;
    b.n_be = be_grid(g);
    b.be_norm = 3.0 * (double)b.nnode;
    b.be_der = ws->be_deriv;
    b.be_ratio = be_weight / (float)b.nnode;
    b.red = ws->red;
    b.xblocks = (int)(((long long)g->ref_dim[1] * g->ref_dim[2] + CONV_X_ROWS - 1) / CONV_X_ROWS);
    return NRB_OK;
}

static int batch_grid(const std::vector<BatchPair>& pairs, long long (*units)(const BatchPair&), int threads,
                      int max_per_sm) {
    long long total = 0;
    for (const BatchPair& b : pairs) total += units(b);
    return grid_for(std::max(1LL, total), threads, max_per_sm);
}

nrb_status launch_batch_be_value(const std::vector<BatchPair>& hp, const BatchPair *d, const OptState *states,
                                 cudaStream_t st) {
    long long units = 0;
    for (const BatchPair& b : hp) units += b.n_be;
    const int grid = (int)std::max(1LL, std::min(units, 2LL * sm_count()));
    KernelTimer timer(TK_BE_VALUE, 0.0, st);
    k_b_be_value<<<grid, 3 * NRB_RED_THREADS, 0, st>>>(d, states, (int)hp.size(), be_basis());
    NRB_CUDA(cudaGetLastError());
    NRB_LAUNCHED("k_b_be_value");
    return NRB_OK;
}

nrb_status launch_batch_node_stage(const std::vector<BatchPair>& hp, const BatchPair *d, const OptState *states,
                                   cudaStream_t st, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join,
                                   nrb_status (*gradient)(const BatchPair *, const OptState *, cudaStream_t, void *),
                                   void *gradient_arg) {
    const int np = (int)hp.size();
    const bool be = hp[0].be_w > 0;
    // bending-energy derivatives on the side branch, beside the voxel passes (they read best only)
    if (be) {
        NRB_CUDA(cudaEventRecord(fork, st));
        NRB_CUDA(cudaStreamWaitEvent(side, fork, 0));
        const int g = batch_grid(hp, [](const BatchPair& b) { return 3 * b.nnode; }, 128, 16);
        KernelTimer timer(TK_BE_GRADIENT, 0.0, side);
        k_b_be_derivatives<<<g, 128, 0, side>>>(d, states, np, be_basis());
        NRB_CUDA(cudaGetLastError());
        NRB_LAUNCHED("k_b_be_derivatives");
    }
    NRB_TRY(gradient(d, states, st, gradient_arg));
    // x pass: shared rows for the widest reference
    int nx = 0, R = 0, nsx = 0;
    long long xb = 0;
    for (const BatchPair& b : hp) {
        nx = std::max(nx, b.rdim[0]);
        R = std::max(R, b.radius[0]);
        nsx = std::max(nsx, b.ns[0]);
        xb += b.xblocks;
    }
    const size_t smem = ((size_t)3 * CONV_X_ROWS * nx + 2 * R + 1 + nsx) * 4;
    if (smem > 227 * 1024) return fail(NRB_ERR_UNSUPPORTED, "convolution: rows and kernel exceed shared memory");
    NRB_CUDA(cudaFuncSetAttribute(k_b_conv_x, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per = 0;
    NRB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_b_conv_x, CONV_X_THREADS, smem));
    const int xg = (int)std::max(1LL, std::min(xb, (long long)std::max(1, per) * sm_count()));
    {
    KernelTimer timer(TK_CONV, 0.0, st);
    k_b_conv_x<<<xg, CONV_X_THREADS, smem, st>>>(d, states, np);
    NRB_CUDA(cudaGetLastError());
    NRB_LAUNCHED("k_b_conv_x");
    const int gy = batch_grid(hp, [](const BatchPair& b) { return 3LL * b.rdim[2] * b.ns[1] * b.ns[0]; }, 256, 16);
    k_b_conv_y<<<gy, 256, 0, st>>>(d, states, np);
    NRB_CUDA(cudaGetLastError());
    NRB_LAUNCHED("k_b_conv_y");
    const int gz = batch_grid(hp, [](const BatchPair& b) { return 3LL * b.ns[2] * b.ns[1] * b.ns[0]; }, 256, 16);
    k_b_conv_z<<<gz, 256, 0, st>>>(d, states, np);
    NRB_CUDA(cudaGetLastError());
    NRB_LAUNCHED("k_b_conv_z");
    const int gn = batch_grid(hp, [](const BatchPair& b) { return b.nnode; }, 256, 16);
    k_b_nodes<<<gn, 256, 0, st>>>(d, states, np);
    NRB_CUDA(cudaGetLastError());
    NRB_LAUNCHED("k_b_nodes");
    }
    if (be) {
        NRB_CUDA(cudaEventRecord(join, side));
        NRB_CUDA(cudaStreamWaitEvent(st, join, 0));
        const int g = batch_grid(hp, [](const BatchPair& b) { return 3 * b.nnode; }, 128, 16);
        KernelTimer timer2(TK_BE_GRADIENT, 0.0, st);
        k_b_be_accumulate<<<g, 128, 0, st>>>(d, states, np, be_basis());
        NRB_CUDA(cudaGetLastError());
        NRB_LAUNCHED("k_b_be_accumulate");
    }
    return NRB_OK;
}
}  // namespace nrb

extern "C" nrb_status nrb_approx_bending_energy_gradient(nrb_workspace *ws, const nrb_geometry *g,
                                                         const float *cpp, float weight, float *node_grad,
                                                         void *stream) {
    if (!ws || !g || !cpp || !node_grad) return fail(NRB_ERR_INVALID, "nrb_approx_bending_energy_gradient: null pointer");
    cudaStream_t st = as_stream(stream);
    NRB_TRY(launch_be_derivatives(ws, g, cpp, st));
    return launch_be_accumulate(ws, g, weight, node_grad, st);
}

// fred holds two partial arrays of NRB_RED_BLOCKS floats (min | max)
static nrb_status rescale_impl(float *img, int64_t n, float lo, float hi, float *fred, cudaStream_t st) {
    const int np = (int)std::max<long long>(1, std::min<long long>((n + NRB_RED_THREADS - 1) / NRB_RED_THREADS, NRB_RED_BLOCKS));
    k_minmax<<<np, NRB_RED_THREADS, 0, st>>>(n, img, fred, fred + NRB_RED_BLOCKS);
    NRB_LAUNCHED("k_minmax");
    k_rescale<<<grid_for(n, 256), 256, 0, st>>>(n, img, fred, fred + NRB_RED_BLOCKS, np, lo, hi);
    NRB_LAUNCHED("k_rescale");
    return NRB_OK;
}

namespace nrb {
nrb_status rescale_with(float *img, int64_t n, float lo, float hi, float *fred, cudaStream_t st) {
    return rescale_impl(img, n, lo, hi, fred, st);
}
}  // namespace nrb

extern "C" nrb_status nrb_intensity_rescale(float *img, int64_t nvox_, float new_min, float new_max, void *stream) {
    if (!img || nvox_ <= 0) return fail(NRB_ERR_INVALID, "nrb_intensity_rescale: bad argument");
    cudaStream_t st = as_stream(stream);
    float *fred = nullptr;
    NRB_CUDA(tmp_alloc(&fred, 2 * NRB_RED_BLOCKS * sizeof(float), st));
    NRB_TRY(rescale_impl(img, nvox_, new_min, new_max, fred, st));
    NRB_CUDA(cudaFreeAsync(fred, st));
    return NRB_OK;
}

extern "C" nrb_status nrb_get_maximal_length(const float *node_grad, int64_t nnode, nrb_objective *obj,
                                             double *max_host, void *stream) {
    if (!node_grad || nnode <= 0) return fail(NRB_ERR_INVALID, "nrb_get_maximal_length: bad argument");
    cudaStream_t st = as_stream(stream);
    const int np = (int)std::max<long long>(1, std::min<long long>((nnode + NRB_RED_THREADS - 1) / NRB_RED_THREADS, NRB_RED_BLOCKS));
    float *pm = nullptr;
    double *dm = nullptr;
    NRB_CUDA(tmp_alloc(&pm, np * sizeof(float), st));
    NRB_CUDA(tmp_alloc(&dm, sizeof(double), st));
    k_maxlen<<<np, NRB_RED_THREADS, 0, st>>>(nnode, node_grad, pm);
    NRB_LAUNCHED("k_maxlen");
    k_maxlen_finish<<<1, 32, 0, st>>>(pm, np, obj, dm);
    NRB_LAUNCHED("k_maxlen_finish");
    if (max_host) {
        NRB_CUDA(cudaMemcpyAsync(max_host, dm, sizeof(double), cudaMemcpyDeviceToHost, st));
        NRB_CUDA(cudaStreamSynchronize(st));
    }
    NRB_CUDA(cudaFreeAsync(pm, st));
    NRB_CUDA(cudaFreeAsync(dm, st));
    return NRB_OK;
}

namespace nrb {
// max length into obj->max_grad_len then normalisation by it, scratch from the workspace
// UpdateGradientValues with the first-call branch taken on the device (flag read at run time)
nrb_status cg_update_flagged(nrb_workspace *ws, float *grad, float *g1, float *g2, int64_t n, const int *first_call,
                             cudaStream_t st) {
    const int np = (int)std::max<long long>(1, std::min<long long>((n + NRB_RED_THREADS - 1) / NRB_RED_THREADS, NRB_RED_BLOCKS));
    k_cg_dots<<<np, NRB_RED_THREADS, 0, st>>>(n, grad, g1, g2, ws->red);
    NRB_LAUNCHED("k_cg_dots");
    k_cg_update<<<grid_for(n, 256), 256, 0, st>>>(n, grad, g1, g2, ws->red, np, first_call);
    NRB_LAUNCHED("k_cg_update");
    return NRB_OK;
}

nrb_status max_and_normalise(nrb_workspace *ws, float *grad, int64_t nnode, nrb_objective *obj, cudaStream_t st) {
    const int np = (int)std::max<long long>(1, std::min<long long>((nnode + NRB_RED_THREADS - 1) / NRB_RED_THREADS, NRB_RED_BLOCKS));
    k_maxlen<<<np, NRB_RED_THREADS, 0, st>>>(nnode, grad, ws->fred);
    NRB_LAUNCHED("k_maxlen");
    k_maxlen_finish<<<1, 32, 0, st>>>(ws->fred, np, obj, nullptr);
    NRB_LAUNCHED("k_maxlen_finish");
    k_normalise<<<grid_for(3 * nnode, 256), 256, 0, st>>>(3 * nnode, grad, obj, -1.0);
    NRB_LAUNCHED("k_normalise");
    return NRB_OK;
}
}  // namespace nrb

extern "C" nrb_status nrb_normalise_gradient(float *node_grad, int64_t nnode, double max_len,
                                             const nrb_objective *obj, void *stream) {
    if (!node_grad || nnode <= 0 || (max_len < 0 && !obj))
        return fail(NRB_ERR_INVALID, "nrb_normalise_gradient: bad argument");
    k_normalise<<<grid_for(3 * nnode, 256), 256, 0, as_stream(stream)>>>(3 * nnode, node_grad, obj, max_len);
    NRB_LAUNCHED("k_normalise");
    return NRB_OK;
}

extern "C" nrb_status nrb_update_control_point_position(float *cur, const float *best, const float *grad,
                                                        float scale, int64_t n, void *stream) {
    if (!cur || !best || !grad || n <= 0) return fail(NRB_ERR_INVALID, "nrb_update_control_point_position: bad argument");
    k_update<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(n, cur, best, grad, scale);
    NRB_LAUNCHED("k_update");
    return NRB_OK;
}

extern "C" nrb_status nrb_conjugate_gradient(nrb_workspace *ws, float *grad, float *g1, float *g2, int64_t n,
                                             int first_call, void *stream) {
    if (!ws || !grad || !g1 || !g2 || n <= 0) return fail(NRB_ERR_INVALID, "nrb_conjugate_gradient: bad argument");
    cudaStream_t st = as_stream(stream);
    if (first_call) {
        k_cg_init<<<grid_for(n, 256), 256, 0, st>>>(n, grad, g1, g2);
        NRB_LAUNCHED("k_cg_init");
        return NRB_OK;
    }
    const int np = (int)std::max<long long>(1, std::min<long long>((n + NRB_RED_THREADS - 1) / NRB_RED_THREADS, NRB_RED_BLOCKS));
    k_cg_dots<<<np, NRB_RED_THREADS, 0, st>>>(n, grad, g1, g2, ws->red);
    NRB_LAUNCHED("k_cg_dots");
    k_cg_update<<<grid_for(n, 256), 256, 0, st>>>(n, grad, g1, g2, ws->red, np, nullptr);
    NRB_LAUNCHED("k_cg_update");
    return NRB_OK;
}

// ---------------------------------------------------------------------------------------------
// pyramid and grid helpers used by the registration driver
// ---------------------------------------------------------------------------------------------
namespace nrb {

// Gaussian smoothing of reg_downsampleImage (sigma = -0.7355 voxel, all three axes in one
// reg_tools_kernelConvolution call, density normalised once at the end), then nearest-neighbour
// downsampling. tmp needs 4 * nvox(in) floats.
nrb_status smooth_and_downsample(const float *in, const int32_t idim[3], float *out, const int32_t odim[3],
                                 const float new_xyz[16], const float old_ijk[16], float *tmp, cudaStream_t st) {
    const double temp = 0.7355;  // |sigma|, voxel units
    const int radius = (int)(temp * 3.0f);
    std::vector<float> k(2 * radius + 1);
    for (int i = -radius; i <= radius; ++i)
        k[radius + i] = (float)(std::exp(-(double)(i * i) / (2.0 * temp * temp)) / (temp * 2.506628274631));
    float *dk = nullptr;
    NRB_CUDA(tmp_alloc(&dk, k.size() * 4, st));
    NRB_CUDA(cudaMemcpyAsync(dk, k.data(), k.size() * 4, cudaMemcpyHostToDevice, st));
    const long long nv = nvox(idim);
    float *v0 = tmp, *d0 = tmp + nv, *v1 = tmp + 2 * nv, *d1 = tmp + 3 * nv;
    const int g = grid_for(nv, 256);
    k_conv_axis<<<g, 256, 0, st>>>(idim[0], idim[1], idim[2], 0, in, nullptr, dk, radius, v0, d0);
    NRB_LAUNCHED("k_conv_axis");
    k_conv_axis<<<g, 256, 0, st>>>(idim[0], idim[1], idim[2], 1, v0, d0, dk, radius, v1, d1);
    NRB_LAUNCHED("k_conv_axis");
    k_conv_axis<<<g, 256, 0, st>>>(idim[0], idim[1], idim[2], 2, v1, d1, dk, radius, v0, d0);
    NRB_LAUNCHED("k_conv_axis");
    k_conv_normalise<<<g, 256, 0, st>>>(nv, in, v0, d0, v1);
    NRB_LAUNCHED("k_conv_normalise");
    const long long no = nvox(odim);
    k_downsample<<<grid_for(no, 256), 256, 0, st>>>(odim[0], odim[1], odim[2], idim[0], idim[1], idim[2],
                                                    to_mat34(new_xyz), to_mat34(old_ijk), v1, out);
    NRB_LAUNCHED("k_downsample");
    NRB_CUDA(cudaFreeAsync(dk, st));
    return NRB_OK;
}

nrb_status grid_identity(const int32_t cdim[3], const float cxyz[16], float *cpp, cudaStream_t st) {
    const long long nc = nvox(cdim);
    k_grid_identity<<<grid_for(nc, 256), 256, 0, st>>>(cdim[0], cdim[1], cdim[2], to_mat34(cxyz), cpp);
    NRB_LAUNCHED("k_grid_identity");
    return NRB_OK;
}

nrb_status grid_refine(const int32_t odim[3], const float *old, const int32_t ndim[3], float *out, cudaStream_t st) {
    const long long nc = nvox(ndim);
    k_grid_refine<<<grid_for(nc, 256), 256, 0, st>>>(odim[0], odim[1], odim[2], ndim[0], ndim[1], ndim[2], old, out);
    NRB_LAUNCHED("k_grid_refine");
    return NRB_OK;
}

}  // namespace nrb
