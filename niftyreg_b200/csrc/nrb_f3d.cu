// Whole F3D registration on the device: the pyramid, per-level grid refinement and the
// conjugate-gradient line search of reg_f3d<float>::Run, with every image, grid and optimiser
// array resident in HBM. Each objective evaluation returns one packed struct to the host, which
// takes the line-search branch exactly as Optimiser::Optimise does.
#include <cooperative_groups.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <vector>

#include "nrb_state.cuh"

namespace cg = cooperative_groups;

namespace nrb {

// defined in nrb_ops.cu
nrb_status smooth_and_downsample(const float *in, const int32_t idim[3], float *out, const int32_t odim[3],
                                 const float new_xyz[16], const float old_ijk[16], float *tmp, cudaStream_t st);
nrb_status grid_identity(const int32_t cdim[3], const float cxyz[16], float *cpp, cudaStream_t st);
nrb_status grid_refine(const int32_t odim[3], const float *old, const int32_t ndim[3], float *out, cudaStream_t st);
nrb_status rescale_with(float *img, int64_t n, float lo, float hi, float *fred, cudaStream_t st);
nrb_status max_and_normalise(nrb_workspace *ws, float *grad, int64_t nnode, nrb_objective *obj, cudaStream_t st);
nrb_status cg_update_flagged(nrb_workspace *ws, float *grad, float *g1, float *g2, int64_t n, const int *first_call,
                             cudaStream_t st);

// ---------------------------------------------------------------------------------------------
// Device-resident optimiser: the state of ConjugateGradient<float>::Optimise and of the level
// loop of reg_base::Run (reg-lib/Optimiser.cpp:129-173, reg-lib/_reg_base.cpp:760-800), kept in
// device memory and advanced by single-thread control kernels, so a whole level runs as one
// CUDA graph whose two WHILE nodes (iterations, line-search steps) read conditions the control
// kernels set. The arithmetic on the step lengths and objective values is the host loop's,
// operation for operation.
// ---------------------------------------------------------------------------------------------

__global__ void k_ctl_level(OptState *s, OptState init, cudaGraphConditionalHandle outer) {
    *s = init;
    cudaGraphSetConditional(outer, outer_continues(init) ? 1u : 0u);
}

// after GetObjectiveFunctionGradient: iteration counted; current_size = min(current_size, max_step)
__global__ void k_ctl_gradient_done(OptState *s) {
    s->it += 1;
    s->n_grad += 1;
    s->current_size = s->max_step < s->current_size ? s->max_step : s->current_size;
}

// Optimiser::Optimise entry (after UpdateGradientValues consumed first_call)
__global__ void k_ctl_line_start(OptState *s, cudaGraphConditionalHandle inner) {
    s->first_call = 0;
    s->line_iter = 0;
    s->added_len = 0.f;
    s->cur_len = s->current_size;
    cudaGraphSetConditional(inner, line_continues(*s) ? 1u : 0u);
}

// end of Optimise (start length = added length) and the restart rule of _reg_base.cpp:784-793
__global__ void k_ctl_line_end(OptState *s, cudaGraphConditionalHandle outer) {
    cudaGraphSetConditional(outer, line_end(s) ? 1u : 0u);
}

// The node-grid tail of a gradient evaluation in one launch (one cluster of TAIL_CTAS blocks):
// GetMaximalLength + NormaliseGradient (reg-lib/Compute.cpp:140-176), the iteration count and
// min(current_size, max_step), ConjugateGradient::UpdateGradientValues (reg-lib/Optimiser.cpp:
// 231-317) and the start of Optimise. Every value is computed with the operations, and every
// FP64 dot product with the partition and summation order, of the separate kernels the host loop
// launches (k_maxlen/k_maxlen_finish, k_normalise, k_cg_dots/k_cg_update), so both loops stay
// bit-identical. n = 3 * nnode; partials: 2 * NRB_RED_BLOCKS doubles.
constexpr int TAIL_CTAS = 8, TAIL_THREADS = 1024;
constexpr long long kNodeTailMaxNodes = 16384;  // above it the passes are bandwidth-bound on 8 SMs

// The cluster's work: returns the largest node-gradient length; the optimiser state is only read
// (first_call) and the caller publishes the rest.
__device__ __forceinline__ double node_tail_cluster(cg::cluster_group& cluster, long long nnode, float *__restrict__ g,
                                                    float *__restrict__ g1, float *__restrict__ g2,
                                                    double *__restrict__ partials, const OptState *__restrict__ s) {
    __shared__ float fmx[TAIL_THREADS / 32];
    __shared__ double red[TAIL_THREADS];
    __shared__ double gam_s;
    const int rank = (int)cluster.block_rank(), tid = threadIdx.x;
    const long long gtid = (long long)rank * TAIL_THREADS + tid, gstride = (long long)TAIL_CTAS * TAIL_THREADS;
    const long long n = 3 * nnode;
    const bool first = s->first_call != 0;  // read before block 0 changes the state at the end
    // largest node-gradient length (a max: exact in any order)
    float mx = 0.f;
    for (long long i = gtid; i < nnode; i += gstride) {
        const float x = g[i], y = g[nnode + i], z = g[2 * nnode + i];
        mx = fmaxf(mx, sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z))));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((tid & 31) == 0) fmx[tid >> 5] = mx;
    __syncthreads();
    if (tid == 0) {
        float m = 0.f;
        for (int w = 0; w < TAIL_THREADS / 32; ++w) m = fmaxf(m, fmx[w]);
        fmx[0] = m;
    }
    cluster.sync();
    float m = 0.f;
#pragma unroll
    for (int q = 0; q < TAIL_CTAS; ++q) m = fmaxf(m, cluster.map_shared_rank(fmx, q)[0]);
    const double len = (double)m;
    const bool scale = len != 0;
    const double inv = scale ? 1.0 / len : 1.0;
    auto normalised = [&](long long i) { return scale ? (float)((double)g[i] * inv) : g[i]; };
    if (first) {
        for (long long i = gtid; i < n; i += gstride) {
            const float v = normalised(i);
            g[i] = v;
            g1[i] = -v;
            g2[i] = -v;
        }
    } else {
        // the FP64 dots of k_cg_dots: virtual blocks of NRB_RED_THREADS threads, grid-stride over
        // np virtual blocks, tree-summed per virtual block
        const long long nb = (n + NRB_RED_THREADS - 1) / NRB_RED_THREADS;
        const int np = (int)(nb < 1 ? 1 : (nb > NRB_RED_BLOCKS ? NRB_RED_BLOCKS : nb));
        constexpr int VPB = TAIL_THREADS / NRB_RED_THREADS;  // virtual blocks per block at a time
        const int vsub = tid / NRB_RED_THREADS, t = tid % NRB_RED_THREADS;
        double *r = red + vsub * NRB_RED_THREADS;
        for (int v0 = rank * VPB; v0 < np; v0 += TAIL_CTAS * VPB) {  // same trip count in the block
            const int v = v0 + vsub;
            double gg = 0, dgg = 0;
            if (v < np)
                for (long long i = (long long)v * NRB_RED_THREADS + t; i < n; i += (long long)np * NRB_RED_THREADS) {
                    const float gi = normalised(i);
                    gg += (double)__fmul_rn(g2[i], g1[i]);
                    dgg += (double)__fmul_rn(__fadd_rn(gi, g1[i]), gi);
                }
            // block_sum_d's tree, once for gg and once for dgg
            r[t] = gg;
            __syncthreads();
            for (int k = NRB_RED_THREADS / 2; k > 0; k >>= 1) {
                if (t < k) r[t] += r[t + k];
                __syncthreads();
            }
            const double a = r[0];
            __syncthreads();
            r[t] = dgg;
            __syncthreads();
            for (int k = NRB_RED_THREADS / 2; k > 0; k >>= 1) {
                if (t < k) r[t] += r[t + k];
                __syncthreads();
            }
            if (t == 0 && v < np) {
                partials[2 * v] = a;
                partials[2 * v + 1] = r[0];
            }
            __syncthreads();
        }
        cluster.sync();  // every partial written
        if (rank == 0 && tid == 0) {
            double gg = 0, dgg = 0;
            for (int i = 0; i < np; ++i) {
                gg += partials[2 * i];
                dgg += partials[2 * i + 1];
            }
            gam_s = dgg / gg;
        }
        cluster.sync();
        const double gm = *cluster.map_shared_rank(&gam_s, 0);
        for (long long i = gtid; i < n; i += gstride) {
            const float a1 = -normalised(i);
            const float a2 = (float)((double)a1 + gm * (double)g2[i]);
            g1[i] = a1;
            g2[i] = a2;
            g[i] = -a2;
        }
    }
    return len;
}

__global__ void __cluster_dims__(TAIL_CTAS, 1, 1) __launch_bounds__(TAIL_THREADS)
k_node_tail(long long nnode, float *__restrict__ g, float *__restrict__ g1, float *__restrict__ g2,
            double *__restrict__ partials, nrb_objective *__restrict__ obj, OptState *__restrict__ s,
            cudaGraphConditionalHandle line) {
    cg::cluster_group cluster = cg::this_cluster();
    const double len = node_tail_cluster(cluster, nnode, g, g1, g2, partials, s);
    if (cluster.block_rank() == 0 && threadIdx.x == 0) {
        obj->max_grad_len = len;
        // iteration counted, current_size = min(current_size, max_step), then Optimise starts
        cudaGraphSetConditional(line, gradient_done_line_start(s) ? 1u : 0u);
    }
    cluster.sync();  // block 0's shared values stay readable until every block has read them
}

// One node-tail cluster per pair (cluster q = pair q) for the pairs in GRAD: the same work, then
// the pair's line search starts (LINE), or ends at once when it has no step to take (GRAD again
// after a restart, or DONE); the last cluster sets whether the level goes on.
__global__ void __cluster_dims__(TAIL_CTAS, 1, 1) __launch_bounds__(TAIL_THREADS)
k_b_node_tail(const BatchPair *__restrict__ pairs, OptState *__restrict__ states, int npairs,
              BatchCtl *__restrict__ bctl, int in_graph, cudaGraphConditionalHandle outer) {
    cg::cluster_group cluster = cg::this_cluster();
    const int p = blockIdx.x / TAIL_CTAS;
    if (states[p].phase == PH_GRAD) {
        const BatchPair& B = pairs[p];
        OptState *s = &states[p];
        const double len = node_tail_cluster(cluster, B.nnode, B.grad, B.g1, B.g2, B.red, s);
        if (cluster.block_rank() == 0 && threadIdx.x == 0) {
            B.obj->max_grad_len = len;
            const bool line = gradient_done_line_start(s);
            s->phase = line ? PH_LINE : (line_end(s) ? PH_GRAD : PH_DONE);
        }
        cluster.sync();
    }
    if (cluster.block_rank() != 0) return;
    if (!batch_last_cluster(&bctl->ticket_tail, gridDim.x / TAIL_CTAS)) return;
    int nline, ngrad;
    batch_counts(states, npairs, nline, ngrad);
    if (threadIdx.x == 0) {
        if (in_graph) cudaGraphSetConditional(outer, nline + ngrad > 0 ? 1u : 0u);
        bctl->go_on = nline + ngrad > 0;
    }
}

// StoreCurrentDof after an accepted step: best = best + (-len) * grad, the trial position the
// objective kernel formed on the fly (same float operations)
__global__ void k_accept(long long n, float *__restrict__ best, const float *__restrict__ grad,
                         const OptState *__restrict__ s) {
    pdl_wait();  // the decision comes from the finalize
    if (!s->accepted) return;
    const float scale = -s->step_len;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        best[i] = __fadd_rn(best[i], __fmul_rn(scale, grad[i]));
}

int elementwise_grid(long long n) {
    return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 4LL * 148));
}

// dst = the dense [nz][ny][nx] volume src in the middle of a [nz+2m][ny+2m][nx+2m] one whose
// margin holds `value`
__global__ void k_pad_volume(const float *__restrict__ src, int nx, int ny, int nz, int m, float value,
                             float *__restrict__ dst) {
    const int px = nx + 2 * m, py = ny + 2 * m;
    const long long n = (long long)px * py * (nz + 2 * m);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % px) - m;
        const long long r = i / px;
        const int y = (int)(r % py) - m;
        const int z = (int)(r / py) - m;
        const bool in = x >= 0 && x < nx && y >= 0 && y < ny && z >= 0 && z < nz;
        dst[i] = in ? src[((long long)z * ny + y) * nx + x] : value;
    }
}

nrb_status pad_volume(const float *src, const int32_t dim[3], int margin, float value, float *dst,
                      const float **origin, cudaStream_t st) {
    k_pad_volume<<<elementwise_grid(padded_voxels(dim, margin)), 256, 0, st>>>(src, dim[0], dim[1], dim[2], margin,
                                                                              value, dst);
    NRB_LAUNCHED("k_pad_volume");
    *origin = dst + ((long long)margin * (dim[1] + 2 * margin) + margin) * (dim[0] + 2 * margin) + margin;
    return NRB_OK;
}

struct GraphHolder {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~GraphHolder() {
        if (exec) cudaGraphExecDestroy(exec);
        if (g) cudaGraphDestroy(g);
    }
};

// Appends a WHILE node driven by `h` to the graph `st` is capturing, after everything captured
// so far, and returns its body graph; capture then continues after the node.
nrb_status capture_while(cudaStream_t st, cudaGraphConditionalHandle h, cudaGraph_t *body) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t capg = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    NRB_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &capg, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) return fail(NRB_ERR_CUDA, "registration: stream capture not active");
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    NRB_CUDA(cudaGraphAddNode(&node, capg, deps, nd, &cp));
    *body = cp.conditional.phGraph_out[0];
    NRB_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    return NRB_OK;
}

// Appends an IF node driven by `h` (body runs when the handle is non-zero), like capture_while.
nrb_status capture_if(cudaStream_t st, cudaGraphConditionalHandle h, cudaGraph_t *body) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t capg = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    NRB_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &capg, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) return fail(NRB_ERR_CUDA, "registration: stream capture not active");
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    NRB_CUDA(cudaGraphAddNode(&node, capg, deps, nd, &cp));
    *body = cp.conditional.phGraph_out[0];
    NRB_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    return NRB_OK;
}

namespace {

// Ceil<int>(float) and the like of reg-lib/cpu/Maths.hpp:63-85
int ceil_ref(float x) {
    const int i = (int)x;
    return i + (x > (float)i);
}

// Voxel <-> mm of an image with identity orientation and origin `origin` (qform code 1, no
// sform): qto_xyz = diag(pixdim) + origin, qto_ijk its inverse (nifti_mat44_inverse rounds the
// double-precision inverse to float).
// inverse of an affine voxel <-> mm matrix, in double (nifti_mat44_inverse's role)
static bool affine_inverse(const float m[16], float out[16]) {
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

// Geometry of one image of the registration. An image whose voxel -> mm matrix is the spacing
// on the diagonal keeps that form (the arithmetic of an identity orientation with an origin);
// any other orientation is held in full in `m`. `sform`: the matrix came from an sform, whose
// columns reg_createControlPointGrid scales for the grid (the qform's are rebuilt instead).
struct Header {
    int32_t dim[3];
    float pixdim[3];
    float origin[3];
    bool full = false, sform = false;
    float m[16];
    void xyz(float out[16]) const {
        if (full) {
            memcpy(out, m, 16 * sizeof(float));
            return;
        }
        float *m = out;
        memset(m, 0, 16 * sizeof(float));
        for (int i = 0; i < 3; ++i) {
            m[5 * i] = pixdim[i];
            m[4 * i + 3] = origin[i];
        }
        m[15] = 1.f;
    }
    void ijk(float out[16]) const {
        if (full) {
            affine_inverse(m, out);
            return;
        }
        float *m = out;
        memset(m, 0, 16 * sizeof(float));
        for (int i = 0; i < 3; ++i) {
            const double inv = 1.0 / (double)pixdim[i];
            m[5 * i] = (float)inv;
            m[4 * i + 3] = (float)(-(double)origin[i] * inv);
        }
        m[15] = 1.f;
    }
    int64_t n() const { return (int64_t)dim[0] * dim[1] * dim[2]; }
};

// An input image's geometry: dims, spacings and, when given, its voxel -> mm matrix (from an
// sform when `sform`). Without a matrix the image has the identity orientation at origin 0.
struct ImageDesc {
    int32_t dim[3];
    float pixdim[3];
    const float *xyz = nullptr;
    bool sform = false;
};

static Header header_of(const ImageDesc& d) {
    Header h{};
    for (int i = 0; i < 3; ++i) {
        h.dim[i] = d.dim[i];
        h.pixdim[i] = d.pixdim[i];
        h.origin[i] = 0.f;
    }
    if (d.xyz) {
        const float *m = d.xyz;
        const bool plain = m[1] == 0.f && m[2] == 0.f && m[4] == 0.f && m[6] == 0.f && m[8] == 0.f && m[9] == 0.f &&
                           m[0] == d.pixdim[0] && m[5] == d.pixdim[1] && m[10] == d.pixdim[2];
        if (plain) {
            h.origin[0] = m[3];
            h.origin[1] = m[7];
            h.origin[2] = m[11];
        } else {
            h.full = true;
            memcpy(h.m, m, 12 * sizeof(float));
            h.m[12] = h.m[13] = h.m[14] = 0.f;
            h.m[15] = 1.f;
        }
        h.sform = d.sform;
    }
    return h;
}

// reg_downsampleImage's header (reg-lib/cpu/_reg_tools.cpp:1344-1417): every axis whose size / 2
// is at least 32 halves (ceil) and doubles its spacing and its matrix column (exact in float);
// the origin stays
static Header halve(const Header& src) {
    Header dst = src;
    for (int i = 0; i < 3; ++i) {
        const bool down = src.dim[i] / 2 >= 32;
        dst.dim[i] = down && src.dim[i] > 1 ? ceil_ref((float)(src.dim[i] / 2.0)) : src.dim[i];
        dst.pixdim[i] = down ? src.pixdim[i] * 2.0f : src.pixdim[i];
        if (down && src.full)
            for (int r = 0; r < 3; ++r) dst.m[4 * r + i] = src.m[4 * r + i] * 2.0f;
    }
    return dst;
}

// The control-point grid of reg_createControlPointGrid / reg_spline_refineControlPointGrid
// (reg-lib/cpu/_reg_localTrans.cpp:21-128, 1860-1925) over reference `r` with spacing `s` mm:
// ceil(n * d / s + 3) nodes per axis, the reference's orientation (an sform's columns scaled by
// the float ratio s / d; a qform's rebuilt with spacing s), the origin shifted by one node
// (Mat44Mul of (-1, -1, -1), in double).
static Header grid_header(const Header& r, const float s[3]) {
    Header g{};
    for (int i = 0; i < 3; ++i) {
        g.dim[i] = ceil_ref((float)r.dim[i] * r.pixdim[i] / s[i] + 3.f);
        g.pixdim[i] = s[i];
        g.origin[i] = (float)((double)s[i] * -1.0 + (double)r.origin[i]);
    }
    if (!r.full && !r.sform) return g;
    float rm[16];
    r.xyz(rm);
    g.full = true;
    g.sform = r.sform;
    for (int j = 0; j < 3; ++j) {
        if (r.sform) {
            const float ratio = s[j] / r.pixdim[j];
            for (int i = 0; i < 3; ++i) g.m[4 * i + j] = rm[4 * i + j] * ratio;
        } else {
            for (int i = 0; i < 3; ++i) g.m[4 * i + j] = (float)((double)rm[4 * i + j] / r.pixdim[j] * s[j]);
        }
    }
    for (int i = 0; i < 3; ++i)
        g.m[4 * i + 3] = (float)((double)g.m[4 * i] * -1.0 + (double)g.m[4 * i + 1] * -1.0 +
                                 (double)g.m[4 * i + 2] * -1.0 + (double)rm[4 * i + 3]);
    g.m[12] = g.m[13] = g.m[14] = 0.f;
    g.m[15] = 1.f;
    return g;
}

// Every buffer of a registration is allocated and freed in the order of the registration's
// stream, so concurrent registrations on other streams never wait for each other's frees.
struct DevBuf {
    float *p = nullptr;
    cudaStream_t st = nullptr;
    ~DevBuf() { dev_free(p, st); }
    nrb_status alloc(size_t n, cudaStream_t s) {
        dev_free(p, st);
        p = nullptr;
        st = s;
        if (dev_alloc(&p, std::max<size_t>(n, 1) * sizeof(float), st) != cudaSuccess) {
            cudaGetLastError();
            return fail(NRB_ERR_OOM, "registration: device allocation failed");
        }
        return NRB_OK;
    }
};

struct NmiHandle {
    nrb_nmi *h = nullptr;
    ~NmiHandle() { nrb_nmi_destroy(h); }
};
struct WsHandle {
    nrb_workspace *h = nullptr;
    ~WsHandle() { nrb_workspace_destroy(h); }
};

// reg_createImagePyramid for both images (definition below the registration class)
nrb_status build_pyramids(const float *ref, const float *flo, const ImageDesc& rd, const ImageDesc& fd, int levels,
                          cudaStream_t st, std::vector<Header>& hdr, std::vector<Header>& fhdr,
                          std::vector<DevBuf>& ref_pyr, std::vector<DevBuf>& flo_pyr);

// reg_f3d<float> with the NMI measure and the bending-energy penalty on the B200 platform.
class F3dRegistration {
public:
    F3dRegistration(const nrb_f3d_params& p, cudaStream_t st): p_(p), st_(st) {}

    // warped_out (optional, host or device): the floating image warped by the final grid with
    // cubic-spline interpolation (reg_f3d::GetWarpedImage), reference-sized
    nrb_status Run(const float *ref, const float *flo, const ImageDesc& rd, const ImageDesc& fd, float *cpp_out,
                   int64_t cap, nrb_f3d_result *res, float *warped_out = nullptr);
    const Header& grid() const { return grid_; }

    // The pieces of Run a batched driver calls for every pair: Begin (pyramid, grid, budget);
    // per level PrepareLevel (InitLevel without the initial objective), Describe (the pair's
    // BatchPair and starting optimiser state), Absorb (the optimiser state the batched level
    // ended with), EndLevel; then Finish.
    nrb_status Begin(const float *ref, const float *flo, const ImageDesc& rd, const ImageDesc& fd);
    nrb_status PrepareLevel(int level, float& max_step) {
        batched_ = true;
        return InitLevel(level, max_step);
    }
    nrb_status Describe(float max_step, BatchPair& b, OptState& init);
    nrb_status Absorb(const OptState& out);
    void EndLevel() { max_it_ /= 2; }
    nrb_status Finish(const float *flo, float *cpp_out, int64_t cap, nrb_f3d_result *res, float *warped_out = nullptr);

private:
    // reg_f3d::GetObjectiveFunctionValue (_reg_f3d.cpp:443-462)
    nrb_status GetObjectiveFunctionValue(double& value) {
        nrb_objective o;
        NRB_TRY(f3d_objective(ws_.h, nmi_.h, &g_, ref_.p, flo_org_, margin_, nullptr, cur_.p, pad_, sim_w_, be_w_,
                              obj_, &o, st_));
        cur_w_measure_ = sim_w_ > 0 ? (double)sim_w_ * o.nmi : 0.0;
        cur_w_be_ = be_w_ > 0 ? (double)be_w_ * o.be : 0.0;
        cur_nmi_ = o.nmi;
        cur_be_ = o.be;
        ++n_obj_;
        value = cur_w_measure_ - cur_w_be_;
        return NRB_OK;
    }
    // reg_f3d::GetObjectiveFunctionGradient (_reg_f3d.cpp:553-576) + NormaliseGradient (:395-410)
    nrb_status GetObjectiveFunctionGradient() {
        NRB_TRY(f3d_gradient(ws_.h, nmi_.h, &g_, ref_.p, flo_org_, margin_, nullptr, cur_.p, pad_, sim_w_, be_w_,
                             vgrad_.p, grad_.p, st_));
        ++it_;
        ++n_grad_;
        return max_and_normalise(ws_.h, grad_.p, nc_, obj_, st_);
    }
    void UpdateBestObjFunctionValue() {
        best_w_measure_ = cur_w_measure_;
        best_w_be_ = cur_w_be_;
        best_nmi_ = cur_nmi_;
        best_be_ = cur_be_;
    }
    nrb_status StoreCurrentDof() {
        NRB_CUDA(cudaMemcpyAsync(best_.p, cur_.p, 3 * nc_ * sizeof(float), cudaMemcpyDeviceToDevice, st_));
        return NRB_OK;
    }
    nrb_status RestoreBestDof() {
        NRB_CUDA(cudaMemcpyAsync(cur_.p, best_.p, 3 * nc_ * sizeof(float), cudaMemcpyDeviceToDevice, st_));
        return NRB_OK;
    }
    // ConjugateGradient::Optimise = UpdateGradientValues + Optimiser::Optimise
    // (reg-lib/Optimiser.cpp:320-323, :129-173)
    nrb_status Optimise(float max_length, float small_length, float& start_length) {
        NRB_TRY(nrb_conjugate_gradient(ws_.h, grad_.p, g1_.p, g2_.p, 3 * nc_, first_call_ ? 1 : 0, st_));
        first_call_ = false;
        size_t line_iteration = 0;
        float added_length = 0;
        float current_length = start_length;
        while (current_length > small_length && line_iteration < 12 && it_ < max_it_) {
            NRB_TRY(nrb_update_control_point_position(cur_.p, best_.p, grad_.p, -current_length, 3 * nc_, st_));
            double value = 0;
            NRB_TRY(GetObjectiveFunctionValue(value));
            if (value > best_obj_) {
                UpdateBestObjFunctionValue();
                best_obj_ = value;
                added_length += current_length;
                current_length *= 1.1f;
                current_length = std::min(current_length, max_length);
                NRB_TRY(StoreCurrentDof());
            } else {
                current_length *= 0.5;
            }
            ++it_;
            ++line_iteration;
        }
        start_length = added_length;
        return RestoreBestDof();
    }

    // the level loop of reg_base::Run on the host (one synchronising read per evaluation)
    nrb_status RunLevelHost(float max_step, float smallest_size, float current_size) {
        bool just_restarted = false;
        while (current_size) {
            if (it_ >= max_it_) break;
            NRB_TRY(GetObjectiveFunctionGradient());
            current_size = std::min(current_size, max_step);
            NRB_TRY(Optimise(max_step, smallest_size, current_size));
            if (p_.verbose)
                printf("[nrb] [%zu] objective %.6f = (wSIM)%.6f - (wBE)%.6g [+ %g mm]\n", it_, best_obj_,
                       best_w_measure_, best_w_be_, current_size);
            // _reg_base.cpp:784-793: one restart to steepest descent on a stalled line search
            if (current_size == 0) {
                if (!just_restarted && it_ < max_it_) {
                    first_call_ = true;
                    current_size = max_step;
                    just_restarted = true;
                }
            } else {
                just_restarted = false;
            }
        }
        return NRB_OK;
    }
    nrb_status RunLevelGraph(float max_step, float smallest_size, float current_size);
    nrb_status CaptureGradient(cudaStream_t cs);
    nrb_status CaptureLineStep(cudaStream_t cs, cudaGraphConditionalHandle line);

    nrb_status BuildPyramid(const float *ref, const float *flo, const ImageDesc& rd, const ImageDesc& fd);
    nrb_status CreateGrid();
    nrb_status InitLevel(int level, float& max_step);

    nrb_f3d_params p_;
    cudaStream_t st_;
    int levels_ = 0;
    std::vector<Header> hdr_, fhdr_;  // reference and floating pyramids
    std::vector<DevBuf> ref_pyr_, flo_pyr_;
    // current level
    nrb_geometry g_{};
    DevBuf ref_, flo_, vgrad_, grad_, best_, g1_, g2_, cur_;
    // the floating image as the voxel passes read it: flo_org_ is its voxel (0, 0, 0), inside
    // flo_pad_ (a copy with margin_ voxels of padding values on every side) or flo_ (margin 0)
    DevBuf flo_pad_;
    FloTexture ftex_;  // flo_pad_ as a layered texture (p_.floating_texture)
    const float *flo_org_ = nullptr;
    int margin_ = 0;
    NmiHandle nmi_;
    WsHandle ws_;
    nrb_objective *obj_ = nullptr;
    int64_t nc_ = 0;
    // grid
    Header grid_{};
    float pad_ = std::numeric_limits<float>::quiet_NaN();
    float sim_w_ = 1, be_w_ = 0;
    float spacing_mm_[3] = { 0, 0, 0 };
    // optimiser state
    size_t it_ = 0, max_it_ = 0;
    bool first_call_ = true;
    double best_obj_ = 0;
    double cur_w_measure_ = 0, cur_w_be_ = 0, best_w_measure_ = 0, best_w_be_ = 0;
    double cur_nmi_ = 0, cur_be_ = 0, best_nmi_ = 0, best_be_ = 0;
    int64_t n_obj_ = 0, n_grad_ = 0;
    std::chrono::steady_clock::time_point t0_;
    bool batched_ = false;  // levels driven by a batched graph (the initial objective is its first stage)
    // device-resident optimiser
    bool graph_ok_ = true;
    OptState *dstate_ = nullptr;
    cudaStream_t cap_st_ = nullptr;

public:
    ~F3dRegistration() {
        flo_texture_release(ftex_);
        dev_free(dstate_, st_);
        if (cap_st_) cudaStreamDestroy(cap_st_);
    }
    void UseGraphs(bool on) { graph_ok_ = on; }
};

// GetObjectiveFunctionGradient as captured launches: the fused gradient (nrb_f3d_gradient's
// sequence), then NormaliseGradient. In the graph the current position is never materialised:
// after every line search it equals the best one (RestoreBestDof), which the gradient reads
// directly. The reference recomputes the joint histogram at that position first
// (_reg_nmi.cpp:625); here the NMI tables of the best position are still resident (the table
// sets alternate between evaluations), and they are the same numbers.
nrb_status F3dRegistration::CaptureGradient(cudaStream_t cs) {
    nrb_workspace *ws = ws_.h;
    const bool be = be_w_ > 0;
    if (be) {
        NRB_TRY(fork_side(ws, cs));
        NRB_TRY(launch_be_derivatives(ws, &g_, best_.p, ws->side));
    }
    NRB_TRY(launch_fused_gradient(ws, nmi_.h, &g_, ref_.p, flo_org_, nullptr, best_.p, pad_, 1.0, vgrad_.p, cs, dstate_,
                                  margin_));
    NRB_TRY(launch_convolve_to_nodes(ws, &g_, vgrad_.p, sim_w_, grad_.p, cs));
    if (be) {
        NRB_TRY(join_side(ws, cs));
        NRB_TRY(launch_be_accumulate(ws, &g_, be_w_, grad_.p, cs));
    }
    return NRB_OK;  // the node-grid tail follows as one launch (k_node_tail)
}

// One line-search step as captured launches: the objective at the trial position
// best - cur_len * grad formed inside the kernels (UpdateControlPointPosition fused away), the
// bending energy of the same position beside it on the side stream, and the finalize taking the
// step (value, acceptance, next length, WHILE condition) and storing an accepted trial position
// into best. (One launch per step, the finalize run by the objective's last cluster to finish,
// was measured slower: a launch of 8-block clusters holds fewer blocks at once and paid a fixed
// cost of about 18 us per step at the coarse levels.)
nrb_status F3dRegistration::CaptureLineStep(cudaStream_t cs, cudaGraphConditionalHandle line) {
    nrb_workspace *ws = ws_.h;
    int n_be = 0;
    if (be_w_ > 0) {
        NRB_TRY(fork_side(ws, cs));
        NRB_TRY(launch_be_value(ws, &g_, best_.p, ws->side, grad_.p, dstate_));
        n_be = be_partial_count(&g_);
    }
    NRB_TRY(launch_fused_objective(ws, nmi_.h, &g_, ref_.p, flo_org_, nullptr, best_.p, pad_, cs, grad_.p, dstate_,
                                   margin_));
    if (be_w_ > 0) NRB_TRY(join_side(ws, cs));
    const long long n = 3 * nc_;
    // small grids: the finalize also stores an accepted trial position (one launch fewer per
    // step); large grids: a whole-device pass does it
    const bool fold = nc_ <= kNodeTailMaxNodes;
    NRB_TRY(launch_nmi_finalize(nmi_.h, ws->be_partials, n_be, 3 * nvox(g_.cpp_dim), sim_w_, be_w_, obj_, cs,
                                dstate_, line, fold ? best_.p : nullptr, grad_.p, fold ? n : 0));
    if (fold) return NRB_OK;
    NRB_CUDA(launch_pdl(true, k_accept, dim3(elementwise_grid(n)), dim3(256), 0, cs, n, best_.p, grad_.p,
                        (const OptState *)dstate_));
    NRB_LAUNCHED("k_accept");
    return NRB_OK;
}

// One level of reg_base::Run as one CUDA graph:
//   level init -> WHILE(iterations) { gradient, CG direction, line start,
//                                     WHILE(line search) { update, objective, step, store },
//                                     line end + restart rule, restore best }
// launched once; the host reads the optimiser state back when it ends.
nrb_status F3dRegistration::RunLevelGraph(float max_step, float smallest_size, float current_size) {
    const auto t_enter = std::chrono::steady_clock::now();
    if (!cap_st_) NRB_CUDA(cudaStreamCreateWithFlags(&cap_st_, cudaStreamNonBlocking));
    if (!dstate_) NRB_CUDA(dev_alloc(&dstate_, sizeof(OptState), st_));
    const long long n = 3 * nc_;
    OptState init = {};
    init.best_obj = best_obj_;
    init.best_w_measure = best_w_measure_;
    init.best_w_be = best_w_be_;
    init.best_nmi = best_nmi_;
    init.best_be = best_be_;
    init.it = (long long)it_;
    init.max_it = (long long)max_it_;
    init.n_obj = n_obj_;
    init.n_grad = n_grad_;
    init.current_size = current_size;
    init.max_step = max_step;
    init.small_step = smallest_size;
    init.first_call = first_call_ ? 1 : 0;
    init.best_buf = 0;  // the level's initial evaluation wrote the first table set

    GraphHolder top;
    cudaGraph_t outer_body = nullptr, inner_body = nullptr;
    cudaGraphConditionalHandle h_outer, h_inner;
    NRB_CUDA(cudaGraphCreate(&top.g, 0));
    NRB_CUDA(cudaGraphConditionalHandleCreate(&h_outer, top.g, 0, 0));
    const long long c0 = g_launch_count.load();
    auto abort_capture = [&](nrb_status s) {
        cudaGraph_t dummy = nullptr;
        cudaStreamEndCapture(cap_st_, &dummy);
        cudaGetLastError();
        return s;
    };
    // top level
    NRB_CUDA(cudaStreamBeginCaptureToGraph(cap_st_, top.g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    k_ctl_level<<<1, 1, 0, cap_st_>>>(dstate_, init, h_outer);
    if (cudaGetLastError() != cudaSuccess) return abort_capture(fail(NRB_ERR_CUDA, "registration: level init launch"));
    g_launch_count.fetch_add(1);
    {
        nrb_status s = capture_while(cap_st_, h_outer, &outer_body);
        if (s != NRB_OK) return abort_capture(s);
    }
    NRB_CUDA(cudaStreamEndCapture(cap_st_, &top.g));
    const long long c_top = g_launch_count.load() - c0;
    // one iteration
    NRB_CUDA(cudaGraphConditionalHandleCreate(&h_inner, outer_body, 0, 0));
    NRB_CUDA(cudaStreamBeginCaptureToGraph(cap_st_, outer_body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    {
        nrb_status s = CaptureGradient(cap_st_);
        if (nc_ <= kNodeTailMaxNodes) {
            // small grids: the node-grid tail is a chain of latency-bound launches; one cluster
            // does all of it
            if (s == NRB_OK) {
                k_node_tail<<<TAIL_CTAS, TAIL_THREADS, 0, cap_st_>>>(nc_, grad_.p, g1_.p, g2_.p, ws_.h->red, obj_,
                                                                     dstate_, h_inner);
                g_launch_count.fetch_add(1);
                if (cudaGetLastError() != cudaSuccess) s = fail(NRB_ERR_CUDA, "registration: node tail launch");
            }
        } else {
            // large grids: the separate kernels spread the passes over the whole device
            if (s == NRB_OK) s = max_and_normalise(ws_.h, grad_.p, nc_, obj_, cap_st_);
            if (s == NRB_OK) {
                k_ctl_gradient_done<<<1, 1, 0, cap_st_>>>(dstate_);
                g_launch_count.fetch_add(1);
                if (cudaGetLastError() != cudaSuccess) s = fail(NRB_ERR_CUDA, "registration: gradient count launch");
            }
            if (s == NRB_OK) s = cg_update_flagged(ws_.h, grad_.p, g1_.p, g2_.p, n, &dstate_->first_call, cap_st_);
            if (s == NRB_OK) {
                k_ctl_line_start<<<1, 1, 0, cap_st_>>>(dstate_, h_inner);
                g_launch_count.fetch_add(1);
                if (cudaGetLastError() != cudaSuccess) s = fail(NRB_ERR_CUDA, "registration: line start launch");
            }
        }
        if (s == NRB_OK) s = capture_while(cap_st_, h_inner, &inner_body);
        if (s == NRB_OK) {
            k_ctl_line_end<<<1, 1, 0, cap_st_>>>(dstate_, h_outer);
            g_launch_count.fetch_add(1);
            if (cudaGetLastError() != cudaSuccess) s = fail(NRB_ERR_CUDA, "registration: line end launch");
        }
        if (s != NRB_OK) return abort_capture(s);
    }
    NRB_CUDA(cudaStreamEndCapture(cap_st_, &outer_body));
    const long long c_outer = g_launch_count.load() - c0 - c_top;
    // one line-search step
    NRB_CUDA(cudaStreamBeginCaptureToGraph(cap_st_, inner_body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    {
        nrb_status s = CaptureLineStep(cap_st_, h_inner);
        if (s != NRB_OK) return abort_capture(s);
    }
    NRB_CUDA(cudaStreamEndCapture(cap_st_, &inner_body));
    const long long c_inner = g_launch_count.load() - c0 - c_top - c_outer;
    g_launch_count.fetch_sub(c_top + c_outer + c_inner);  // counted again below, per execution

    const auto t_captured = std::chrono::steady_clock::now();
    NRB_CUDA(cudaGraphInstantiate(&top.exec, top.g, 0));
    const auto t_instantiated = std::chrono::steady_clock::now();
    NRB_CUDA(cudaGraphLaunch(top.exec, st_));
    // RestoreBestDof of the last line search: the current position is the best one
    NRB_CUDA(cudaMemcpyAsync(cur_.p, best_.p, n * sizeof(float), cudaMemcpyDeviceToDevice, st_));
    OptState out;
    NRB_CUDA(cudaMemcpyAsync(&out, dstate_, sizeof(OptState), cudaMemcpyDeviceToHost, st_));
    NRB_CUDA(cudaStreamSynchronize(st_));
    if (p_.verbose) {
        const auto t_ran = std::chrono::steady_clock::now();
        auto ms = [](auto a, auto b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
        printf("[nrb]   graph: capture %.3f ms, instantiate %.3f ms, run %.3f ms\n", ms(t_enter, t_captured),
               ms(t_captured, t_instantiated), ms(t_instantiated, t_ran));
    }
    const long long iters = out.n_grad - n_grad_, steps = out.n_obj - n_obj_;
    g_launch_count.fetch_add(c_top + iters * c_outer + steps * c_inner);
    best_obj_ = out.best_obj;
    best_w_measure_ = out.best_w_measure;
    best_w_be_ = out.best_w_be;
    best_nmi_ = out.best_nmi;
    best_be_ = out.best_be;
    it_ = (size_t)out.it;
    n_obj_ = out.n_obj;
    n_grad_ = out.n_grad;
    first_call_ = out.first_call != 0;
    if (p_.verbose)
        printf("[nrb] level done: %lld iterations, objective %.6f = (wSIM)%.6f - (wBE)%.6g\n", (long long)it_,
               best_obj_, best_w_measure_, best_w_be_);
    return NRB_OK;
}

// reg_createImagePyramid (reg-lib/cpu/_reg_tools.cpp:1705-1733): the finest level is the input,
// each coarser level halves (ceil) every axis whose current size / 2 is at least 32, after a
// Gaussian smoothing.
nrb_status build_pyramids(const float *ref, const float *flo, const ImageDesc& rd, const ImageDesc& fd, int levels,
                          cudaStream_t st, std::vector<Header>& hdr, std::vector<Header>& fhdr,
                          std::vector<DevBuf>& ref_pyr, std::vector<DevBuf>& flo_pyr) {
    hdr.assign(levels, Header{});
    fhdr.assign(levels, Header{});
    ref_pyr = std::vector<DevBuf>(levels);
    flo_pyr = std::vector<DevBuf>(levels);
    hdr[levels - 1] = header_of(rd);
    fhdr[levels - 1] = header_of(fd);
    const Header& rf = hdr[levels - 1];
    const Header& ff = fhdr[levels - 1];
    NRB_TRY(ref_pyr[levels - 1].alloc(rf.n(), st));
    NRB_TRY(flo_pyr[levels - 1].alloc(ff.n(), st));
    NRB_CUDA(cudaMemcpyAsync(ref_pyr[levels - 1].p, ref, rf.n() * 4, cudaMemcpyDefault, st));
    NRB_CUDA(cudaMemcpyAsync(flo_pyr[levels - 1].p, flo, ff.n() * 4, cudaMemcpyDefault, st));
    if (levels == 1) return NRB_OK;
    DevBuf tmp;
    NRB_TRY(tmp.alloc(4 * std::max(rf.n(), ff.n()), st));
    for (int l = levels - 2; l >= 0; --l) {
        // each image halves along its own axes
        hdr[l] = halve(hdr[l + 1]);
        fhdr[l] = halve(fhdr[l + 1]);
        float nxyz[16], oijk[16];
        NRB_TRY(ref_pyr[l].alloc(hdr[l].n(), st));
        hdr[l].xyz(nxyz);
        hdr[l + 1].ijk(oijk);
        NRB_TRY(smooth_and_downsample(ref_pyr[l + 1].p, hdr[l + 1].dim, ref_pyr[l].p, hdr[l].dim, nxyz, oijk, tmp.p,
                                      st));
        NRB_TRY(flo_pyr[l].alloc(fhdr[l].n(), st));
        fhdr[l].xyz(nxyz);
        fhdr[l + 1].ijk(oijk);
        NRB_TRY(smooth_and_downsample(flo_pyr[l + 1].p, fhdr[l + 1].dim, flo_pyr[l].p, fhdr[l].dim, nxyz, oijk,
                                      tmp.p, st));
    }
    return NRB_OK;  // tmp is freed in stream order
}

// The pair's description for a batched level (its walks, buffers, NMI tables, node stage) and
// the optimiser state its level starts from (RunLevelGraph's init, the initial objective still
// to be evaluated: phase INIT).
nrb_status F3dRegistration::Describe(float max_step, BatchPair& b, OptState& init) {
    if (!(sim_w_ > 0)) return fail(NRB_ERR_UNSUPPORTED, "batched registration: the similarity weight must be > 0");
    memset(&b, 0, sizeof(b));
    NRB_TRY(batch_walks(ws_.h, nmi_.h, &g_, pad_, margin_, b.wo, b.wg));
    b.ref = ref_.p;
    b.flo = flo_org_;
    b.best = best_.p;
    b.grad = grad_.p;
    b.g1 = g1_.p;
    b.g2 = g2_.p;
    b.vgrad = vgrad_.p;
    b.hist = nmi_.h->hist;
    b.pro0 = nmi_.h->pro;
    b.logt0 = nmi_.h->logt;
    b.last0 = nmi_.h->last;
    b.pro1 = nmi_.h->pro2;
    b.logt1 = nmi_.h->logt2;
    b.last1 = nmi_.h->last2;
    b.obj = obj_;
    b.rb = nmi_.h->rb;
    b.fb = nmi_.h->fb;
    NRB_TRY(batch_node_stage(ws_.h, &g_, sim_w_, be_w_, b));
    b.sim_w = sim_w_;
    b.be_w = be_w_;
    b.obj_items = b.wo.nitems;
    b.grad_items = b.wg.nitems;
    init = OptState{};
    init.it = (long long)it_;
    init.max_it = (long long)max_it_;
    init.n_obj = n_obj_;
    init.n_grad = n_grad_;
    init.current_size = max_step;
    init.max_step = max_step;
    init.small_step = max_step / 100.0f;
    init.first_call = 1;
    init.best_buf = 0;
    init.phase = PH_INIT;
    return NRB_OK;
}

// the optimiser state a batched level ended with; RestoreBestDof (current = best)
nrb_status F3dRegistration::Absorb(const OptState& out) {
    best_obj_ = out.best_obj;
    best_w_measure_ = out.best_w_measure;
    best_w_be_ = out.best_w_be;
    best_nmi_ = out.best_nmi;
    best_be_ = out.best_be;
    it_ = (size_t)out.it;
    n_obj_ = out.n_obj;
    n_grad_ = out.n_grad;
    first_call_ = out.first_call != 0;
    NRB_CUDA(cudaMemcpyAsync(cur_.p, best_.p, 3 * nc_ * sizeof(float), cudaMemcpyDeviceToDevice, st_));
    return NRB_OK;
}

nrb_status F3dRegistration::BuildPyramid(const float *ref, const float *flo, const ImageDesc& rd,
                                         const ImageDesc& fd) {
    return build_pyramids(ref, flo, rd, fd, levels_, st_, hdr_, fhdr_, ref_pyr_, flo_pyr_);
}

// reg_f3d::Initialise (_reg_f3d.cpp:161-200) -> reg_createControlPointGrid
// (reg-lib/cpu/_reg_localTrans.cpp:21-128) on the coarsest reference.
nrb_status F3dRegistration::CreateGrid() {
    const Header& r = hdr_[0];
    float spacing[3];
    for (int i = 0; i < 3; ++i) {
        float s = p_.spacing[i];
        if (s != s) s = p_.spacing[0];
        spacing_mm_[i] = s < 0 ? s * -hdr_[levels_ - 1].pixdim[i] : s;
        spacing[i] = spacing_mm_[i] * powf(2.f, (float)(levels_ - 1));
    }
    grid_ = grid_header(r, spacing);
    float cxyz[16];
    grid_.xyz(cxyz);
    NRB_TRY(cur_.alloc(3 * grid_.n(), st_));
    return grid_identity(grid_.dim, cxyz, cur_.p, st_);
}

// reg_f3d::InitCurrentLevel (_reg_f3d.cpp:92-132) + InitialiseSimilarity + SetOptimiser
nrb_status F3dRegistration::InitLevel(int level, float& max_step) {
    const Header& r = hdr_[level];
    const Header& fh = fhdr_[level];
    max_step = r.pixdim[0] > r.pixdim[1] ? r.pixdim[0] : r.pixdim[1];
    max_step = r.pixdim[2] > max_step ? r.pixdim[2] : max_step;
    if (level == 0) {
        be_w_ = be_w_ / powf(16.f, (float)(levels_ - 1));
    } else {
        be_w_ = be_w_ * 16.f;
        // reg_spline_refineControlPointGrid onto this level's reference
        const float half[3] = { grid_.pixdim[0] / 2.0f, grid_.pixdim[1] / 2.0f, grid_.pixdim[2] / 2.0f };
        const Header ng = grid_header(r, half);
        DevBuf refined;
        NRB_TRY(refined.alloc(3 * ng.n(), st_));
        NRB_TRY(grid_refine(grid_.dim, cur_.p, ng.dim, refined.p, st_));
        std::swap(cur_.p, refined.p);
        grid_ = ng;
    }
    // content of this level
    nrb_geometry& g = g_;
    for (int i = 0; i < 3; ++i) {
        g.ref_dim[i] = r.dim[i];
        g.ref_pixdim[i] = r.pixdim[i];
        g.flo_dim[i] = fh.dim[i];
        g.flo_pixdim[i] = fh.pixdim[i];
        g.cpp_dim[i] = grid_.dim[i];
        g.cpp_pixdim[i] = grid_.pixdim[i];
    }
    r.xyz(g.ref_xyz);
    r.ijk(g.ref_ijk);
    fh.xyz(g.flo_xyz);
    fh.ijk(g.flo_ijk);
    grid_.xyz(g.cpp_xyz);
    grid_.ijk(g.cpp_ijk);
    nc_ = grid_.n();
    std::swap(ref_.p, ref_pyr_[level].p);
    std::swap(flo_.p, flo_pyr_[level].p);
    ref_.st = flo_.st = st_;
    NRB_TRY(vgrad_.alloc(3 * r.n(), st_));
    NRB_TRY(grad_.alloc(3 * nc_, st_));
    NRB_TRY(best_.alloc(3 * nc_, st_));
    NRB_TRY(g1_.alloc(3 * nc_, st_));
    NRB_TRY(g2_.alloc(3 * nc_, st_));
    nrb_workspace_destroy(ws_.h);
    ws_.h = nullptr;
    NRB_TRY(workspace_create_on(&g_, st_, &ws_.h));
    if (!nmi_.h) NRB_TRY(nmi_create_on(p_.ref_bins + 4, p_.flo_bins + 4, st_, &nmi_.h));
    // reg_nmi::InitialiseMeasure: rescale both images to [2, bins - 3]
    NRB_TRY(rescale_with(ref_.p, r.n(), 2.f, (float)(p_.ref_bins + 4) - 3.f, ws_.h->fred, st_));
    NRB_TRY(rescale_with(flo_.p, fh.n(), 2.f, (float)(p_.flo_bins + 4) - 3.f, ws_.h->fred, st_));
    // the floating image with a margin of padding values, which the voxel passes sample without
    // clamping; the dense copy is released
    margin_ = p_.floating_margin;
    if (margin_ > 0) {
        NRB_TRY(flo_pad_.alloc(padded_voxels(fh.dim, margin_), st_));
        NRB_TRY(pad_volume(flo_.p, fh.dim, margin_, pad_, flo_pad_.p, &flo_org_, st_));
        dev_free(flo_.p, flo_.st);
        flo_.p = nullptr;
        // the padded copy as a layered texture: the fused passes gather its 2x2 footprints (a
        // margin of 2 or more keeps every clamped footprint inside the padding)
        if (p_.floating_texture && margin_ >= 2) {
            const int w = fh.dim[0] + 2 * margin_, h = fh.dim[1] + 2 * margin_, l = fh.dim[2] + 2 * margin_;
            flo_texture_release(ftex_);
            NRB_TRY(flo_texture_acquire(w, h, l, ftex_));
            NRB_TRY(flo_texture_upload(ftex_, flo_pad_.p, w, h, l, st_));
            ws_.h->flo_tex = ftex_.tex;
        }
    } else {
        flo_org_ = flo_.p;
    }
    // ConjugateGradient::Initialise: best = current, objective at the starting point (in a
    // batched level the first stage of the level's graph evaluates it)
    it_ = 0;
    first_call_ = true;
    NRB_TRY(StoreCurrentDof());
    if (batched_) {
        // the batched kernels take each pair's z-chunk from the walk table when its shape has
        // been tuned (their block heights are fixed)
        if (p_.autotune) autotune_lookup(ws_.h, nmi_.h, nullptr, margin_, true);
        return NRB_OK;
    }
    double v = 0;
    NRB_TRY(GetObjectiveFunctionValue(v));
    best_obj_ = v;
    // walk plans for the level: timed once per shape (the evaluation above filled the tables
    // the gradient pass reads); per-launch timing keeps the model's plans
    if (p_.autotune && sim_w_ > 0 && !timing_enabled())
        NRB_TRY(autotune_walks(ws_.h, nmi_.h, &g_, ref_.p, flo_org_, nullptr, cur_.p, pad_, margin_, vgrad_.p, st_));
    return NRB_OK;
}

// reg_f3d::Run up to the level loop: weights, pyramid, grid, iteration budget
nrb_status F3dRegistration::Begin(const float *ref, const float *flo, const ImageDesc& rd, const ImageDesc& fd) {
    t0_ = std::chrono::steady_clock::now();
    levels_ = p_.levels;
    if (levels_ < 1) return fail(NRB_ERR_INVALID, "registration: levels must be >= 1");
    if (p_.ref_bins < 1 || p_.flo_bins < 1) return fail(NRB_ERR_INVALID, "registration: bins must be >= 1");
    if (p_.floating_margin < 0 || p_.floating_margin > 64)
        return fail(NRB_ERR_INVALID, "registration: floating_margin must be in [0, 64]");
    pad_ = p_.padding;
    // reg_f3d::CheckParameters (_reg_f3d.cpp:142-158): weights normalised by the penalty sum
    be_w_ = p_.bending_energy;
    const float penalty = be_w_;
    if (penalty >= 1) {
        sim_w_ = 0;
        be_w_ /= penalty;
    } else {
        sim_w_ = 1 - penalty;
    }
    NRB_CUDA(tmp_alloc(&obj_, sizeof(nrb_objective), st_));
    NRB_CUDA(cudaMemsetAsync(obj_, 0, sizeof(nrb_objective), st_));
    const auto tp = std::chrono::steady_clock::now();
    NRB_TRY(BuildPyramid(ref, flo, rd, fd));
    NRB_TRY(CreateGrid());
    if (p_.verbose) {
        NRB_CUDA(cudaStreamSynchronize(st_));
        printf("[nrb] pyramid and grid %.3f ms\n",
               std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tp).count());
    }
    max_it_ = (size_t)p_.max_iterations;
    max_it_ *= (size_t)std::pow(2, levels_ - 1);
    return NRB_OK;
}

nrb_status F3dRegistration::Run(const float *ref, const float *flo, const ImageDesc& rd, const ImageDesc& fd,
                                float *cpp_out, int64_t cap, nrb_f3d_result *res, float *warped_out) {
    NRB_TRY(Begin(ref, flo, rd, fd));
    for (int level = 0; level < levels_; ++level) {
        float max_step = 0;
        const auto ti = std::chrono::steady_clock::now();
        NRB_TRY(InitLevel(level, max_step));
        if (p_.verbose)
            printf("[nrb] level %d set-up (grid, workspace, rescale, initial objective) %.3f ms\n", level + 1,
                   std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ti).count());
        float current_size = max_step;
        const float smallest_size = max_step / 100.0f;
        UpdateBestObjFunctionValue();
        if (p_.verbose) {
            printf("[nrb] level %d/%d grid %dx%dx%d, initial objective %.6f = (wSIM)%.6f - (wBE)%.6g\n", level + 1,
                   levels_, grid_.dim[0], grid_.dim[1], grid_.dim[2], best_obj_, best_w_measure_, best_w_be_);
            const WalkPlan& wo = ws_.h->walk_obj;
            const WalkPlan& wg = ws_.h->walk_grad;
            printf("[nrb]   walk: objective %d items (z-chunk %d, %lld resident blocks), gradient %d items "
                   "(z-chunk %d, %lld resident blocks)\n", wo.nitems, wo.zchunk,
                   objective_slots(walk_smem_bytes(wo) + (size_t)nmi_.h->rb * nmi_.h->fb * 4), wg.nitems, wg.zchunk,
                   gradient_slots(walk_smem_bytes(wg) + (size_t)nmi_.h->total * 4));
        }
        // the graph path needs a non-zero similarity weight (its gradient has no memset branch)
        // and no per-launch timing; both loops take the same steps
        const auto tl = std::chrono::steady_clock::now();
        const int64_t obj0 = n_obj_, grad0 = n_grad_;
        if (graph_ok_ && sim_w_ > 0 && !timing_enabled()) {
            NRB_TRY(RunLevelGraph(max_step, smallest_size, current_size));
        } else {
            NRB_TRY(RunLevelHost(max_step, smallest_size, current_size));
        }
        if (p_.verbose) {
            NRB_CUDA(cudaStreamSynchronize(st_));
            printf("[nrb] level %d: %lld objective + %lld gradient evaluations in %.2f ms\n", level + 1,
                   (long long)(n_obj_ - obj0), (long long)(n_grad_ - grad0),
                   std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tl).count());
        }
        max_it_ /= 2;
    }
    return Finish(flo, cpp_out, cap, res, warped_out);
}

// reg_f3d::Run after the level loop: the final grid (and warped image) out, the result record
nrb_status F3dRegistration::Finish(const float *flo, float *cpp_out, int64_t cap, nrb_f3d_result *res,
                                   float *warped_out) {
    const int64_t n = 3 * nc_;
    if (cpp_out) {
        if (cap < n) return fail(NRB_ERR_INVALID, "registration: cpp_out capacity too small");
        NRB_CUDA(cudaMemcpyAsync(cpp_out, cur_.p, n * sizeof(float), cudaMemcpyDefault, st_));
    }
    if (warped_out) {
        // reg_f3d::GetWarpedImage: the input floating image (not rescaled) through the final grid
        const Header& rf = hdr_[levels_ - 1];
        const Header& ff = fhdr_[levels_ - 1];
        nrb_geometry wg{};
        for (int i = 0; i < 3; ++i) {
            wg.ref_dim[i] = rf.dim[i];
            wg.ref_pixdim[i] = rf.pixdim[i];
            wg.flo_dim[i] = ff.dim[i];
            wg.flo_pixdim[i] = ff.pixdim[i];
            wg.cpp_dim[i] = grid_.dim[i];
            wg.cpp_pixdim[i] = grid_.pixdim[i];
        }
        rf.xyz(wg.ref_xyz);
        rf.ijk(wg.ref_ijk);
        ff.xyz(wg.flo_xyz);
        ff.ijk(wg.flo_ijk);
        grid_.xyz(wg.cpp_xyz);
        grid_.ijk(wg.cpp_ijk);
        DevBuf fin, wout;
        NRB_TRY(fin.alloc(ff.n(), st_));
        NRB_TRY(wout.alloc(rf.n(), st_));
        NRB_CUDA(cudaMemcpyAsync(fin.p, flo, ff.n() * sizeof(float), cudaMemcpyDefault, st_));
        NRB_TRY(nrb_f3d_warped_image(&wg, fin.p, cur_.p, 3, pad_, wout.p, st_));
        NRB_CUDA(cudaMemcpyAsync(warped_out, wout.p, rf.n() * sizeof(float), cudaMemcpyDefault, st_));
        NRB_CUDA(cudaStreamSynchronize(st_));
    }
    NRB_CUDA(cudaFreeAsync(obj_, st_));
    obj_ = nullptr;
    NRB_CUDA(cudaStreamSynchronize(st_));
    if (res) {
        for (int i = 0; i < 3; ++i) res->cpp_dim[i] = grid_.dim[i];
        res->final_nmi = best_nmi_;
        res->final_be = best_be_;
        res->final_objective = best_obj_;
        res->objective_evaluations = n_obj_;
        res->gradient_evaluations = n_grad_;
        res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
    }
    return NRB_OK;
}

}  // namespace

int64_t registration_footprint(const int32_t dim[3], const float pixdim[3], const nrb_f3d_params *p);

// Raises the release threshold of the library's memory pool to at least `bytes`: the buffers a
// registration frees stay in the pool for the next one instead of being unmapped at every
// synchronisation and mapped again (a measurable share of a registration's time). Never lowers
// it.
static void keep_pool(int64_t bytes) { lib_pool_keep(bytes > 0 ? (uint64_t)bytes : 0); }

// One registration of host or device images on `st` (the entry point of the batch and serving
// drivers, which run several of these concurrently on their own streams).
nrb_status register_on_stream(const float *ref, const float *flo, const int32_t dim[3], const float pixdim[3],
                              const nrb_f3d_params *p, float *cpp_out, int64_t cap, nrb_f3d_result *res,
                              cudaStream_t st) {
    if (st) keep_pool(registration_footprint(dim, pixdim, p));
    F3dRegistration reg(*p, st);
    reg.UseGraphs(p->host_loop == 0);
    ImageDesc d;
    for (int i = 0; i < 3; ++i) {
        d.dim[i] = dim[i];
        d.pixdim[i] = pixdim[i];
    }
    return reg.Run(ref, flo, d, d, cpp_out, cap, res);
}

// Peak device bytes of one registration: the resident pyramid plus the larger of the pyramid
// construction scratch and the finest level's working set (voxel gradient, convolution scratch,
// node arrays, bending-energy derivatives), with slack for the small tables.
int64_t registration_footprint(const int32_t dim[3], const float pixdim[3], const nrb_f3d_params *p) {
    int32_t d[3] = { dim[0], dim[1], dim[2] };
    const int64_t fine = (int64_t)d[0] * d[1] * d[2];
    int64_t pyramid = 0;
    for (int l = 0; l < std::max(1, (int)p->levels); ++l) {
        pyramid += 2 * 4 * (int64_t)d[0] * d[1] * d[2];
        for (int i = 0; i < 3; ++i)
            if (d[i] / 2 >= 32) d[i] = ceil_ref((float)(d[i] / 2.0));
    }
    int64_t nodes = 1;
    for (int i = 0; i < 3; ++i) {
        float s = p->spacing[i];
        if (s != s) s = p->spacing[0];
        const float mm = s < 0 ? s * -pixdim[i] : s;
        nodes *= (int64_t)ceil_ref((float)dim[i] * pixdim[i] / mm + 3.f);
    }
    const int64_t build = 16 * fine;
    const int margin = std::min(64, std::max(0, (int)p->floating_margin));
    const int64_t level = 12 * fine + 24 * fine + (6 * 12 + 72) * nodes + 4 * padded_voxels(dim, margin);
    return pyramid + std::max(build, level) + (4 << 20);
}
}  // namespace nrb

using namespace nrb;

extern "C" void nrb_f3d_default_params(nrb_f3d_params *p) {
    if (!p) return;
    p->levels = 3;
    p->max_iterations = 150;
    p->bending_energy = 0.001f;
    p->spacing[0] = -5.f;
    p->spacing[1] = std::numeric_limits<float>::quiet_NaN();
    p->spacing[2] = std::numeric_limits<float>::quiet_NaN();
    p->ref_bins = 64;
    p->flo_bins = 64;
    p->padding = std::numeric_limits<float>::quiet_NaN();
    p->verbose = 0;
    p->host_loop = 0;
    p->floating_margin = 8;
    p->batch_gradient_percent = 50;
    p->floating_texture = 1;
    p->autotune = 1;
    p->batch_group_mb = 0;
}

extern "C" nrb_status nrb_f3d_grid_dims(const int32_t ref_dim[3], const float ref_pixdim[3], const nrb_f3d_params *p,
                                        int32_t cpp_dim_out[3]) {
    if (!ref_dim || !ref_pixdim || !p || !cpp_dim_out) return fail(NRB_ERR_INVALID, "nrb_f3d_grid_dims: null pointer");
    for (int i = 0; i < 3; ++i) {
        float s = p->spacing[i];
        if (s != s) s = p->spacing[0];
        const float mm = s < 0 ? s * -ref_pixdim[i] : s;
        cpp_dim_out[i] = ceil_ref((float)ref_dim[i] * ref_pixdim[i] / mm + 3.f);
    }
    return NRB_OK;
}

static nrb_status check_register_args(const float *ref, const float *flo, const int32_t dim[3], const float pixdim[3],
                                      const nrb_f3d_params *p) {
    if (!ref || !flo || !dim || !pixdim || !p) return fail(NRB_ERR_INVALID, "registration: null pointer");
    for (int i = 0; i < 3; ++i)
        if (dim[i] < 2 || !(pixdim[i] > 0)) return fail(NRB_ERR_INVALID, "registration: 3D volumes with positive voxel size expected");
    return NRB_OK;
}

extern "C" nrb_status nrb_f3d_register_device(const float *ref, const float *flo, const int32_t dim[3],
                                              const float pixdim[3], const nrb_f3d_params *p, float *cpp_out,
                                              int64_t cpp_capacity, nrb_f3d_result *result, void *stream) {
    NRB_TRY(check_register_args(ref, flo, dim, pixdim, p));
    return register_on_stream(ref, flo, dim, pixdim, p, cpp_out, cpp_capacity, result, as_stream(stream));
}

static nrb_status check_image(const nrb_image *img, const char *what) {
    if (!img || !img->data) return fail(NRB_ERR_INVALID, std::string("registration: null ") + what + " image");
    if (img->nvol != 1) return fail(NRB_ERR_INVALID, std::string("registration: the ") + what + " image must be scalar");
    for (int i = 0; i < 3; ++i)
        if (img->dim[i] < 2 || !(img->pixdim[i] > 0))
            return fail(NRB_ERR_INVALID, std::string("registration: the ") + what +
                                             " image must be 3D with positive voxel sizes");
    return NRB_OK;
}

extern "C" nrb_status nrb_f3d_register_images(const nrb_image *ref, const nrb_image *flo, const nrb_f3d_params *p,
                                              nrb_image *cpp_out, nrb_image *warped_out, nrb_f3d_result *result) {
    NRB_TRY(check_image(ref, "reference"));
    NRB_TRY(check_image(flo, "floating"));
    if (!p || !cpp_out) return fail(NRB_ERR_INVALID, "nrb_f3d_register_images: null pointer");
    memset(cpp_out, 0, sizeof(*cpp_out));
    if (warped_out) memset(warped_out, 0, sizeof(*warped_out));
    ImageDesc rd, fd;
    for (int i = 0; i < 3; ++i) {
        rd.dim[i] = ref->dim[i];
        rd.pixdim[i] = ref->pixdim[i];
        fd.dim[i] = flo->dim[i];
        fd.pixdim[i] = flo->pixdim[i];
    }
    rd.xyz = ref->xyz;
    rd.sform = ref->sform_code > 0;
    fd.xyz = flo->xyz;
    fd.sform = flo->sform_code > 0;
    int32_t cdim[3];
    NRB_TRY(nrb_f3d_grid_dims(ref->dim, ref->pixdim, p, cdim));
    const int64_t ncpp = 3LL * cdim[0] * cdim[1] * cdim[2];
    const int64_t nref = (int64_t)ref->dim[0] * ref->dim[1] * ref->dim[2];
    float *cpp = (float *)malloc((size_t)ncpp * sizeof(float));
    float *warped = warped_out ? (float *)malloc((size_t)nref * sizeof(float)) : nullptr;
    if (!cpp || (warped_out && !warped)) {
        free(cpp);
        free(warped);
        return fail(NRB_ERR_OOM, "nrb_f3d_register_images: host allocation failed");
    }
    const auto t0 = std::chrono::steady_clock::now();
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        free(cpp);
        free(warped);
        return fail(NRB_ERR_CUDA, "nrb_f3d_register_images: stream creation failed");
    }
    const int32_t *big = (int64_t)flo->dim[0] * flo->dim[1] * flo->dim[2] > nref ? flo->dim : ref->dim;
    keep_pool(registration_footprint(big, ref->pixdim, p));
    nrb_status s;
    Header g{};
    {
        F3dRegistration reg(*p, st);
        reg.UseGraphs(p->host_loop == 0);
        s = reg.Run(ref->data, flo->data, rd, fd, cpp, ncpp, result, warped);
        g = reg.grid();
    }
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (s != NRB_OK) {
        free(cpp);
        free(warped);
        return s;
    }
    for (int i = 0; i < 3; ++i) {
        cpp_out->dim[i] = g.dim[i];
        cpp_out->pixdim[i] = g.pixdim[i];
    }
    cpp_out->nvol = 3;
    g.xyz(cpp_out->xyz);
    g.ijk(cpp_out->ijk);
    // the grid carries the reference's form codes (a qform when the reference has none)
    cpp_out->sform_code = ref->sform_code;
    cpp_out->qform_code = ref->sform_code + ref->qform_code > 0 ? ref->qform_code : 1;
    cpp_out->intent_code = 1007;  // NIFTI_INTENT_VECTOR
    cpp_out->intent_p1 = 2.f;     // CUB_SPLINE_GRID
    strncpy(cpp_out->intent_name, "NREG_TRANS", sizeof(cpp_out->intent_name) - 1);
    cpp_out->data = cpp;
    if (warped_out) {
        for (int i = 0; i < 3; ++i) {
            warped_out->dim[i] = ref->dim[i];
            warped_out->pixdim[i] = ref->pixdim[i];
        }
        warped_out->nvol = 1;
        memcpy(warped_out->xyz, ref->xyz, sizeof(ref->xyz));
        memcpy(warped_out->ijk, ref->ijk, sizeof(ref->ijk));
        warped_out->sform_code = ref->sform_code;
        warped_out->qform_code = ref->qform_code;
        warped_out->data = warped;
    }
    if (result) result->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return NRB_OK;
}

extern "C" nrb_status nrb_f3d_register_files(const char *ref_path, const char *flo_path, const nrb_f3d_params *p,
                                             const char *cpp_path, const char *res_path, nrb_f3d_result *result) {
    if (!ref_path || !flo_path || !p || !cpp_path) return fail(NRB_ERR_INVALID, "nrb_f3d_register_files: null pointer");
    nrb_image ref{}, flo{}, cpp{}, warped{};
    nrb_status s = nrb_image_read(ref_path, &ref);
    if (s == NRB_OK) s = nrb_image_read(flo_path, &flo);
    if (s == NRB_OK) s = nrb_f3d_register_images(&ref, &flo, p, &cpp, res_path ? &warped : nullptr, result);
    if (s == NRB_OK) s = nrb_image_write(cpp_path, &cpp);
    if (s == NRB_OK && res_path) s = nrb_image_write(res_path, &warped);
    nrb_image_free(&ref);
    nrb_image_free(&flo);
    nrb_image_free(&cpp);
    nrb_image_free(&warped);
    return s;
}

// ---------------------------------------------------------------------------------------------
// Batched registrations: one graph per pyramid level for every pair of the batch
// ---------------------------------------------------------------------------------------------
// first node of a batched level's graph: the level's WHILE runs (every pair starts in INIT)
__global__ void k_b_level_start(cudaGraphConditionalHandle outer) { cudaGraphSetConditional(outer, 1u); }

namespace {

// Graph construction, instantiation and destruction of batched levels are serialised across
// threads (two server workers each build a graph per level); graph execution is not.
std::mutex g_graph_mu;

// One level of reg_base::Run for every pair, as one CUDA graph:
//   WHILE(any pair active) {
//       [bending-energy value || objective] of the pairs in INIT / LINE, one launch each;
//       finalize, one cluster per pair (tables, NMI, line-search step, accepted step stored,
//       phase moved on; sets the two conditions);
//       IF(enough pairs wait for a gradient, or none has a line-search step left) {
//           [bending-energy derivatives || voxel gradient -> node convolution (4 launches)] ->
//           bending-energy gradient -> node tail, one cluster per pair (CG direction, line
//           search started) } }
// Each launch covers every pair that needs that stage; every pair's arithmetic is its plain
// registration's (same walks, same reductions in the same order), so its result does not depend
// on the rest of the batch. The host syncs once per level.
struct BatchLevelRunner {
    cudaStream_t st = nullptr, cap = nullptr, side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int grad_percent = 50;
    BatchCtl stats{};  // of the last level run
    double graph_ms[2] = { 0, 0 };  // instantiation, execution
    ~BatchLevelRunner() {
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (cap) cudaStreamDestroy(cap);
        if (side) cudaStreamDestroy(side);
    }
    nrb_status init(cudaStream_t s) {
        st = s;
        NRB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        NRB_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
        NRB_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        NRB_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        return NRB_OK;
    }

    nrb_status run(std::vector<BatchPair>& hp, const std::vector<OptState>& init, std::vector<OptState>& out,
                   int64_t *launches) {
        const int np = (int)hp.size();
        BatchLaunch L;
        NRB_TRY(batch_plan(hp, L));
        BatchPair *d_pairs = nullptr;
        OptState *d_states = nullptr;
        BatchCtl *d_ctl = nullptr;
        NRB_CUDA(dev_alloc(&d_pairs, np * sizeof(BatchPair), st));
        NRB_CUDA(dev_alloc(&d_states, np * sizeof(OptState), st));
        NRB_CUDA(dev_alloc(&d_ctl, sizeof(BatchCtl), st));
        BatchCtl ctl{};
        ctl.grad_percent = grad_percent;
        NRB_CUDA(cudaMemcpyAsync(d_pairs, hp.data(), np * sizeof(BatchPair), cudaMemcpyHostToDevice, st));
        NRB_CUDA(cudaMemcpyAsync(d_states, init.data(), np * sizeof(OptState), cudaMemcpyHostToDevice, st));
        NRB_CUDA(cudaMemcpyAsync(d_ctl, &ctl, sizeof(BatchCtl), cudaMemcpyHostToDevice, st));
        nrb_status s = capture_and_run(hp, L, d_pairs, d_states, d_ctl, launches);
        out.resize(np);
        if (s == NRB_OK)
            s = cudaMemcpyAsync(out.data(), d_states, np * sizeof(OptState), cudaMemcpyDeviceToHost, st) == cudaSuccess
                    ? NRB_OK : fail(NRB_ERR_CUDA, "batched level: state read");
        if (s == NRB_OK)
            s = cudaMemcpyAsync(&stats, d_ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, st) == cudaSuccess
                    ? NRB_OK : fail(NRB_ERR_CUDA, "batched level: statistics read");
        dev_free(d_pairs, st);
        dev_free(d_states, st);
        dev_free(d_ctl, st);
        if (s == NRB_OK) NRB_CUDA(cudaStreamSynchronize(st));
        return s;
    }

    // the line-search stage: [bending-energy value || objective] -> finalize
    nrb_status line_stage(std::vector<BatchPair>& hp, const BatchLaunch& L, const BatchPair *d_pairs,
                          OptState *d_states, BatchCtl *d_ctl, cudaStream_t s, bool in_graph,
                          cudaGraphConditionalHandle h_grad, cudaGraphConditionalHandle h_outer, double obj_bytes) {
        const bool be = hp[0].be_w > 0;
        if (be) {
            NRB_CUDA(cudaEventRecord(ev_fork, s));
            NRB_CUDA(cudaStreamWaitEvent(side, ev_fork, 0));
            NRB_TRY(launch_batch_be_value(hp, d_pairs, d_states, side));
            NRB_CUDA(cudaEventRecord(ev_join, side));
        }
        NRB_TRY(launch_batch_objective(d_pairs, d_states, L, s, obj_bytes));
        if (be) NRB_CUDA(cudaStreamWaitEvent(s, ev_join, 0));
        return launch_batch_finalize(d_pairs, d_states, d_ctl, L, in_graph, h_grad, h_outer, s);
    }

    // the gradient stage: [bending-energy derivatives || voxel gradient -> node convolution] ->
    // bending-energy gradient -> node tail
    nrb_status gradient_stage(std::vector<BatchPair>& hp, const BatchLaunch& L, const BatchPair *d_pairs,
                              OptState *d_states, BatchCtl *d_ctl, cudaStream_t s, bool in_graph,
                              cudaGraphConditionalHandle h_outer, double grad_bytes) {
        struct Arg {
            const BatchLaunch *L;
            double bytes;
        } arg{ &L, grad_bytes };
        auto voxels = [](const BatchPair *d, const OptState *states, cudaStream_t st, void *a) {
            const Arg *x = static_cast<const Arg *>(a);
            return launch_batch_gradient(d, states, *x->L, st, x->bytes);
        };
        NRB_TRY(launch_batch_node_stage(hp, d_pairs, d_states, s, side, ev_fork, ev_join, voxels, &arg));
        k_b_node_tail<<<TAIL_CTAS * L.npairs, TAIL_THREADS, 0, s>>>(d_pairs, d_states, L.npairs, d_ctl, in_graph ? 1 : 0,
                                                                  h_outer);
        NRB_CUDA(cudaGetLastError());
        NRB_LAUNCHED("k_b_node_tail");
        return NRB_OK;
    }

    // The level driven from the host, one synchronising read of the decisions per stage (per-
    // kernel timing is on): the same kernels and the same decisions as the graph.
    nrb_status host_driven(std::vector<BatchPair>& hp, const BatchLaunch& L, const BatchPair *d_pairs,
                           OptState *d_states, BatchCtl *d_ctl) {
        const int np = (int)hp.size();
        std::vector<OptState> cur(np);
        for (;;) {
            NRB_CUDA(cudaMemcpyAsync(cur.data(), d_states, np * sizeof(OptState), cudaMemcpyDeviceToHost, st));
            NRB_CUDA(cudaStreamSynchronize(st));
            double ob = 0;
            for (int i = 0; i < np; ++i)
                if (cur[i].phase == PH_INIT || cur[i].phase == PH_LINE)
                    ob += 8.0 * ((double)hp[i].rdim[0] * hp[i].rdim[1] * hp[i].rdim[2]) + 12.0 * (double)hp[i].nnode;
            NRB_TRY(line_stage(hp, L, d_pairs, d_states, d_ctl, st, false, 0, 0, ob));
            BatchCtl c;
            NRB_CUDA(cudaMemcpyAsync(&c, d_ctl, sizeof(c), cudaMemcpyDeviceToHost, st));
            NRB_CUDA(cudaMemcpyAsync(cur.data(), d_states, np * sizeof(OptState), cudaMemcpyDeviceToHost, st));
            NRB_CUDA(cudaStreamSynchronize(st));
            if (c.run_grad) {
                double gb = 0;
                for (int i = 0; i < np; ++i)
                    if (cur[i].phase == PH_GRAD)
                        gb += 20.0 * ((double)hp[i].rdim[0] * hp[i].rdim[1] * hp[i].rdim[2]) + 12.0 * (double)hp[i].nnode;
                NRB_TRY(gradient_stage(hp, L, d_pairs, d_states, d_ctl, st, false, 0, gb));
                NRB_CUDA(cudaMemcpyAsync(&c, d_ctl, sizeof(c), cudaMemcpyDeviceToHost, st));
                NRB_CUDA(cudaStreamSynchronize(st));
            }
            if (!c.go_on) return NRB_OK;
        }
    }

    nrb_status capture_and_run(std::vector<BatchPair>& hp, const BatchLaunch& L, const BatchPair *d_pairs,
                               OptState *d_states, BatchCtl *d_ctl, int64_t *launches) {
        if (timing_enabled()) {
            if (launches) *launches = 0;
            return host_driven(hp, L, d_pairs, d_states, d_ctl);
        }
        std::unique_lock<std::mutex> graph_lock(g_graph_mu);
        GraphHolder top;
        cudaGraph_t while_body = nullptr, if_body = nullptr;
        cudaGraphConditionalHandle h_outer, h_grad;
        NRB_CUDA(cudaGraphCreate(&top.g, 0));
        NRB_CUDA(cudaGraphConditionalHandleCreate(&h_outer, top.g, 0, 0));
        auto abort_capture = [&](nrb_status e) {
            cudaGraph_t dummy = nullptr;
            cudaStreamEndCapture(cap, &dummy);
            if (dummy && dummy != top.g && dummy != while_body && dummy != if_body) cudaGraphDestroy(dummy);
            cudaGetLastError();
            return e;
        };
        const long long c0 = g_launch_count.load();
        NRB_CUDA(cudaStreamBeginCaptureToGraph(cap, top.g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        {
            k_b_level_start<<<1, 1, 0, cap>>>(h_outer);
            nrb_status e = cudaGetLastError() == cudaSuccess ? NRB_OK : fail(NRB_ERR_CUDA, "batched level: start launch");
            if (e == NRB_OK) e = capture_while(cap, h_outer, &while_body);
            if (e != NRB_OK) return abort_capture(e);
        }
        NRB_CUDA(cudaStreamEndCapture(cap, &top.g));
        NRB_CUDA(cudaGraphConditionalHandleCreate(&h_grad, while_body, 0, 0));
        // the line-search stage, then the IF node of the gradient stage
        NRB_CUDA(cudaStreamBeginCaptureToGraph(cap, while_body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        {
            nrb_status e = line_stage(hp, L, d_pairs, d_states, d_ctl, cap, true, h_grad, h_outer, 0.0);
            if (e == NRB_OK) e = capture_if(cap, h_grad, &if_body);
            if (e != NRB_OK) return abort_capture(e);
        }
        NRB_CUDA(cudaStreamEndCapture(cap, &while_body));
        const long long c_line = g_launch_count.load() - c0;
        NRB_CUDA(cudaStreamBeginCaptureToGraph(cap, if_body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        {
            nrb_status e = gradient_stage(hp, L, d_pairs, d_states, d_ctl, cap, true, h_outer, 0.0);
            if (e != NRB_OK) return abort_capture(e);
        }
        NRB_CUDA(cudaStreamEndCapture(cap, &if_body));
        const long long c_grad = g_launch_count.load() - c0 - c_line;
        g_launch_count.fetch_sub(c_line + c_grad);  // counted per execution below
        const auto t_inst = std::chrono::steady_clock::now();
        NRB_CUDA(cudaGraphInstantiate(&top.exec, top.g, 0));
        graph_lock.unlock();
        const auto t_run = std::chrono::steady_clock::now();
        cudaError_t e = cudaGraphLaunch(top.exec, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        graph_lock.lock();  // held while `top` is destroyed on return
        NRB_CUDA(e);
        graph_ms[0] = std::chrono::duration<double, std::milli>(t_run - t_inst).count();
        graph_ms[1] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_run).count();
        if (launches) *launches = c_line + c_grad;
        return NRB_OK;
    }
};

}  // namespace

// Registrations of `n` pairs advanced together, level by level, every stage one launch over the
// pairs that need it. results[i] / cpp_out of pair i equal nrb_f3d_register_host's for pair i
// alone, bit for bit.
nrb_status nrb::register_batch_fused(const nrb_pair *pairs, int n, const nrb_f3d_params *p, nrb_f3d_result *results,
                                cudaStream_t st, int grad_percent) {
    using Clock = std::chrono::steady_clock;
    auto ms_since = [](Clock::time_point t) { return std::chrono::duration<double, std::milli>(Clock::now() - t).count(); };
    const auto t_begin = Clock::now();
    // the stream-ordered pool keeps the whole group's working set between batches (a pool that
    // grows again for every batch pays for mapping the memory each time)
    int64_t group_bytes = 0;
    for (int i = 0; i < n; ++i) group_bytes += registration_footprint(pairs[i].dim, pairs[i].pixdim, p);
    keep_pool(group_bytes);
    std::vector<std::unique_ptr<F3dRegistration>> regs;
    regs.reserve(n);
    for (int i = 0; i < n; ++i) {
        regs.emplace_back(new F3dRegistration(*p, st));
        ImageDesc d;
        for (int k = 0; k < 3; ++k) {
            d.dim[k] = pairs[i].dim[k];
            d.pixdim[k] = pairs[i].pixdim[k];
        }
        NRB_TRY(regs[i]->Begin(pairs[i].ref_host, pairs[i].flo_host, d, d));
    }
    BatchLevelRunner runner;
    runner.grad_percent = grad_percent;
    NRB_TRY(runner.init(st));
    if (p->verbose) {
        NRB_CUDA(cudaStreamSynchronize(st));
        printf("[nrb] batch of %d: pyramids and grids %.2f ms\n", n, ms_since(t_begin));
    }
    for (int level = 0; level < p->levels; ++level) {
        std::vector<BatchPair> hp(n);
        std::vector<OptState> init(n), out;
        const auto t_prep = Clock::now();
        for (int i = 0; i < n; ++i) {
            float max_step = 0;
            NRB_TRY(regs[i]->PrepareLevel(level, max_step));
            NRB_TRY(regs[i]->Describe(max_step, hp[i], init[i]));
        }
        if (p->verbose) {
            NRB_CUDA(cudaStreamSynchronize(st));
            printf("[nrb] batched level %d set-up %.2f ms\n", level + 1, ms_since(t_prep));
        }
        int64_t per_iteration = 0;
        const auto t_level = std::chrono::steady_clock::now();
        NRB_TRY(runner.run(hp, init, out, &per_iteration));
        if (p->verbose) {
            long long evals = 0;
            for (int i = 0; i < n; ++i) evals += out[i].n_obj - init[i].n_obj + out[i].n_grad - init[i].n_grad;
            printf("[nrb] batched level %d: %d pairs, %lld graph iterations, %lld gradient stages, %lld evaluations, "
                   "%.2f ms (graph instantiation %.2f ms, execution %.2f ms)\n", level + 1, n, runner.stats.iterations,
                   runner.stats.grad_stages, evals, ms_since(t_level), runner.graph_ms[0], runner.graph_ms[1]);
        }
        long long iters = 0;
        for (int i = 0; i < n; ++i) {
            iters = std::max(iters, (long long)(out[i].n_obj - init[i].n_obj));
            NRB_TRY(regs[i]->Absorb(out[i]));
            regs[i]->EndLevel();
        }
        g_launch_count.fetch_add(iters * per_iteration);  // an upper bound: the IF stage may be skipped
    }
    const auto t_fin = Clock::now();
    for (int i = 0; i < n; ++i)
        NRB_TRY(regs[i]->Finish(pairs[i].flo_host, pairs[i].cpp_out_host, pairs[i].cpp_capacity,
                                results ? &results[i] : nullptr));
    if (p->verbose) printf("[nrb] batch of %d: results out %.2f ms, total %.2f ms\n", n, ms_since(t_fin), ms_since(t_begin));
    return NRB_OK;
}

extern "C" nrb_status nrb_f3d_register_host(const float *ref_host, const float *flo_host, const int32_t dim[3],
                                            const float pixdim[3], const nrb_f3d_params *p, float *cpp_out_host,
                                            int64_t cpp_capacity, nrb_f3d_result *result) {
    NRB_TRY(check_register_args(ref_host, flo_host, dim, pixdim, p));
    const auto t0 = std::chrono::steady_clock::now();
    cudaStream_t st = nullptr;
    NRB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    nrb_status s;
    // the pyramid's finest level is copied straight from the host buffers
    s = register_on_stream(ref_host, flo_host, dim, pixdim, p, cpp_out_host, cpp_capacity, result, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (s == NRB_OK && result)
        result->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return s;
}

// ---------------------------------------------------------------------------------------------
// F3D2: symmetric registration with stationary velocity fields (reg_f3d2<float>)
// ---------------------------------------------------------------------------------------------
namespace nrb {

nrb_status velocity_to_deformation(const nrb_geometry *g, const float *vel, bool update, int *steps, float *def,
                                   float *fields, float *scratch, unsigned *minmax, cudaStream_t st);
nrb_status exponentiate_gradient(const nrb_geometry *g, const float *vel_other, int steps, float *vgrad,
                                 float *fields, float *scratch, unsigned *minmax, cudaStream_t st);
nrb_status symmetrise_velocity(const int32_t cdim[3], const float fw_xyz[16], float *fw, const float bw_xyz[16],
                               float *bw, cudaStream_t st);

namespace {

// Mat44Mul (reg-lib/cpu/Maths.hpp:271-286): in double, rounded to float
void mat44_mul_f(const float m[16], const float in[3], float out[3]) {
    for (int r = 0; r < 3; ++r)
        out[r] = (float)((double)m[4 * r] * (double)in[0] + (double)m[4 * r + 1] * (double)in[1] +
                         (double)m[4 * r + 2] * (double)in[2] + (double)m[4 * r + 3]);
}

// reg_createSymmetricControlPointGrids (reg-lib/cpu/_reg_localTrans.cpp:133-357) without an
// affine: an axis-aligned grid (sform, identity orientation) over the union of the two images'
// fields of view (corners at voxel 0 and n along each axis), its node 0 one spacing below the
// lowest corner; ceil(extent / spacing + 3) nodes per axis.
Header symmetric_grid_header(const Header& r, const Header& f, const float s[3]) {
    float rm[16], fm[16];
    r.xyz(rm);
    f.xyz(fm);
    float lo[3], hi[3];
    for (int c = 0; c < 8; ++c) {
        const float rc[3] = { (c & 1) ? (float)r.dim[0] : 0.f, (c & 2) ? (float)r.dim[1] : 0.f,
                              (c & 4) ? (float)r.dim[2] : 0.f };
        const float fc[3] = { (c & 1) ? (float)f.dim[0] : 0.f, (c & 2) ? (float)f.dim[1] : 0.f,
                              (c & 4) ? (float)f.dim[2] : 0.f };
        float ro[3], fo[3];
        mat44_mul_f(rm, rc, ro);
        mat44_mul_f(fm, fc, fo);
        for (int i = 0; i < 3; ++i) {
            const float a = std::min(ro[i], fo[i]), b = std::max(ro[i], fo[i]);
            lo[i] = c == 0 ? a : std::min(lo[i], a);
            hi[i] = c == 0 ? b : std::max(hi[i], b);
        }
    }
    Header g{};
    g.full = true;
    g.sform = true;
    memset(g.m, 0, sizeof(g.m));
    for (int i = 0; i < 3; ++i) {
        g.dim[i] = ceil_ref((hi[i] - lo[i]) / s[i] + 3.f);
        g.pixdim[i] = s[i];
        g.m[5 * i] = s[i];
        g.m[4 * i + 3] = lo[i] - s[i];
        g.origin[i] = g.m[4 * i + 3];
    }
    g.m[15] = 1.f;
    return g;
}

// reg_spline_refineControlPointGrid3D without a reference image (_reg_localTrans.cpp:1809-1830,
// 2212-2229): (n - 3) * 2 + 3 nodes, spacing and matrix columns halved, the origin moved to
// node (1, 1, 1) of the halved matrix
Header refine_header(const Header& g) {
    Header n = g;
    float m[16];
    g.xyz(m);
    for (int i = 0; i < 3; ++i) {
        n.dim[i] = (g.dim[i] - 3) * 2 + 3;
        n.pixdim[i] = g.pixdim[i] / 2.0f;
        for (int r = 0; r < 3; ++r) m[4 * r + i] /= 2.f;
    }
    const float one[3] = { 1.f, 1.f, 1.f };
    float o[3];
    mat44_mul_f(m, one, o);
    for (int r = 0; r < 3; ++r) m[4 * r + 3] = o[r];
    n.full = true;
    memcpy(n.m, m, sizeof(m));
    for (int i = 0; i < 3; ++i) n.origin[i] = o[i];
    return n;
}

void fill_geometry(nrb_geometry& g, const Header& r, const Header& f, const Header& c) {
    for (int i = 0; i < 3; ++i) {
        g.ref_dim[i] = r.dim[i];
        g.ref_pixdim[i] = r.pixdim[i];
        g.flo_dim[i] = f.dim[i];
        g.flo_pixdim[i] = f.pixdim[i];
        g.cpp_dim[i] = c.dim[i];
        g.cpp_pixdim[i] = c.pixdim[i];
    }
    r.xyz(g.ref_xyz);
    r.ijk(g.ref_ijk);
    f.xyz(g.flo_xyz);
    f.ijk(g.flo_ijk);
    c.xyz(g.cpp_xyz);
    c.ijk(g.cpp_ijk);
}

// reg_f3d2<float> with the symmetric NMI measure and the bending-energy penalty: forward
// (reference -> floating) and backward velocity grids optimised together by one conjugate
// gradient over both, with the step loop of reg_base::Run on the host.
class F3d2Registration {
public:
    F3d2Registration(const nrb_f3d_params& p, cudaStream_t st): p_(p), st_(st) {}
    // fw_out / bw_out hold cap floats each (3 x the final grid's nodes)
    nrb_status Run(const float *ref, const float *flo, const ImageDesc& rd, const ImageDesc& fd, float *fw_out,
                   float *bw_out, int64_t cap, float *warped_fw, float *warped_bw, nrb_f3d_result *res);
    const Header& grid_fw() const { return gf_; }
    const Header& grid_bw() const { return gb_; }
    int steps() const { return steps_; }

private:
    float *fw(DevBuf& b) { return b.p; }
    float *bw(DevBuf& b) { return b.p + 3 * nc_; }

    nrb_status Fields(int64_t nvox_max) {
        const int64_t need = (int64_t)steps_ * 3 * nvox_max;
        if (need > fields_n_) {
            NRB_TRY(fields_.alloc(need, st_));
            fields_n_ = need;
        }
        return NRB_OK;
    }
    // reg_f3d2::GetDeformationField + WarpFloatingImage (_reg_f3d2.cpp:144-181): the forward
    // field (squaring number updated when the optimiser runs), the backward one with the same
    // number, both images warped (trilinear)
    nrb_status Warp(bool update) {
        NRB_TRY(velocity_to_deformation(&gfw_, fw(cur_), update, &steps_, def_fw_.p, nullptr, scr_r_.p, mm_, st_));
        NRB_TRY(velocity_to_deformation(&gbw_, bw(cur_), false, &steps_, def_bw_.p, nullptr, scr_f_.p, mm_, st_));
        KernelTimer kt(TK_F2_WARP, 0.0, st_);
        NRB_TRY(nrb_resample_image(&gfw_, flo_.p, def_fw_.p, nullptr, pad_, war_fw_.p, st_));
        NRB_TRY(nrb_resample_image(&gbw_, ref_.p, def_bw_.p, nullptr, pad_, war_bw_.p, st_));
        return NRB_OK;
    }
    // both NMI values into the device scalars (obj_[2], obj_[3]); no host read
    nrb_status Similarity() {
        KernelTimer kt(TK_F2_NMI, 0.0, st_);
        NRB_TRY(nrb_nmi_value(nmi_fw_.h, &gfw_, ref_.p, war_fw_.p, nullptr, obj_ + 2, nullptr, st_));
        NRB_TRY(nrb_nmi_value(nmi_bw_.h, &gbw_, flo_.p, war_bw_.p, nullptr, obj_ + 3, nullptr, st_));
        return NRB_OK;
    }
    // reg_f3d2::GetObjectiveFunctionValue (_reg_f3d2.cpp:465-485): both energies and both NMI
    // values land in device scalars and come back in one read
    nrb_status GetObjectiveFunctionValue(bool update, double& value) {
        if (be_w_ > 0) {
            KernelTimer kt(TK_F2_BE, 0.0, st_);
            NRB_TRY(nrb_approx_bending_energy(ws_fw_.h, &gfw_, fw(cur_), obj_, nullptr, st_));
            NRB_TRY(nrb_approx_bending_energy(ws_bw_.h, &gbw_, bw(cur_), obj_ + 1, nullptr, st_));
        }
        if (sim_w_ > 0) {
            NRB_TRY(Warp(update));
            NRB_TRY(Similarity());
        }
        NRB_CUDA(cudaMemcpyAsync(obj_h_, obj_, 4 * sizeof(nrb_objective), cudaMemcpyDeviceToHost, st_));
        NRB_CUDA(cudaStreamSynchronize(st_));
        const double be_f = be_w_ > 0 ? obj_h_[0].be : 0.0, be_b = be_w_ > 0 ? obj_h_[1].be : 0.0;
        const double nf = sim_w_ > 0 ? obj_h_[2].nmi : 0.0, nb = sim_w_ > 0 ? obj_h_[3].nmi : 0.0;
        cur_w_be_ = be_w_ > 0 ? (double)be_w_ * be_f + (double)be_w_ * be_b : 0.0;
        cur_be_ = be_f + be_b;
        cur_nmi_ = nf + nb;
        cur_w_measure_ = sim_w_ > 0 ? (double)sim_w_ * (nf + nb) : 0.0;
        ++n_obj_;
        value = cur_w_measure_ - cur_w_be_;
        return NRB_OK;
    }
    // reg_f3d2::GetObjectiveFunctionGradient (_reg_f3d2.cpp:393-418) with GetVoxelBasedGradient
    // (:244-305), ExponentiateGradient (:637-650) and NormaliseGradient (:369-391)
    nrb_status GetObjectiveFunctionGradient() {
        const int64_t nr = nvox(gfw_.ref_dim), nf = nvox(gbw_.ref_dim);
        if (sim_w_ > 0) {
            // the fields and warped images at the best position: those of the accepted trial when
            // it recomputed the squaring number (the same flow gives the same number, so they are
            // what Warp(true) would compute); else computed here
            if (best_fields_) {
                std::swap(def_fw_.p, bdef_fw_.p);
                std::swap(def_bw_.p, bdef_bw_.p);
                std::swap(war_fw_.p, bwar_fw_.p);
                std::swap(war_bw_.p, bwar_bw_.p);
                steps_ = best_steps_;
                best_fields_ = false;  // the best buffers now hold scratch
            } else {
                NRB_TRY(Warp(true));
            }
            NRB_TRY(Similarity());  // reg_nmi::GetVoxelBasedSimilarityMeasureGradientFw recomputes both
            {
                KernelTimer kt(TK_F2_VOXEL_GRADIENT, 0.0, st_);
                NRB_CUDA(cudaMemsetAsync(vg_fw_.p, 0, 3 * nr * sizeof(float), st_));
                NRB_CUDA(cudaMemsetAsync(vg_bw_.p, 0, 3 * nf * sizeof(float), st_));
                NRB_TRY(nrb_get_image_gradient(&gfw_, flo_.p, def_fw_.p, nullptr, pad_, wg_fw_.p, st_));
                NRB_TRY(nrb_get_image_gradient(&gbw_, ref_.p, def_bw_.p, nullptr, pad_, wg_bw_.p, st_));
                // the FP64 window: the trajectory follows reg_f3d2's
                NRB_TRY(nmi_voxel_gradient(nmi_fw_.h, &gfw_, ref_.p, war_fw_.p, wg_fw_.p, nullptr, 1.0, vg_fw_.p, st_,
                                           true));
                NRB_TRY(nmi_voxel_gradient(nmi_bw_.h, &gbw_, flo_.p, war_bw_.p, wg_bw_.p, nullptr, 1.0, vg_bw_.p, st_,
                                           true));
            }
            // forward gradient along the backward transformation on the reference grid, and back
            NRB_TRY(Fields(std::max(nr, nf)));
            nrb_geometry gx = gfw_;
            for (int i = 0; i < 3; ++i) gx.cpp_dim[i] = gbw_.cpp_dim[i], gx.cpp_pixdim[i] = gbw_.cpp_pixdim[i];
            memcpy(gx.cpp_xyz, gbw_.cpp_xyz, sizeof(gx.cpp_xyz));
            memcpy(gx.cpp_ijk, gbw_.cpp_ijk, sizeof(gx.cpp_ijk));
            NRB_TRY(exponentiate_gradient(&gx, bw(cur_), steps_, vg_fw_.p, fields_.p, scr_r_.p, mm_, st_));
            gx = gbw_;
            for (int i = 0; i < 3; ++i) gx.cpp_dim[i] = gfw_.cpp_dim[i], gx.cpp_pixdim[i] = gfw_.cpp_pixdim[i];
            memcpy(gx.cpp_xyz, gfw_.cpp_xyz, sizeof(gx.cpp_xyz));
            memcpy(gx.cpp_ijk, gfw_.cpp_ijk, sizeof(gx.cpp_ijk));
            NRB_TRY(exponentiate_gradient(&gx, fw(cur_), steps_, vg_bw_.p, fields_.p, scr_f_.p, mm_, st_));
            KernelTimer kt(TK_F2_NODES, 0.0, st_);
            NRB_TRY(nrb_convolve_voxel_based_gradient(ws_fw_.h, &gfw_, vg_fw_.p, sim_w_, fw(grad_), st_));
            NRB_TRY(nrb_convolve_voxel_based_gradient(ws_bw_.h, &gbw_, vg_bw_.p, sim_w_, bw(grad_), st_));
        } else {
            NRB_CUDA(cudaMemsetAsync(grad_.p, 0, 6 * nc_ * sizeof(float), st_));
        }
        ++it_;
        ++n_grad_;
        if (be_w_ > 0) {
            NRB_TRY(nrb_approx_bending_energy_gradient(ws_fw_.h, &gfw_, fw(cur_), be_w_, fw(grad_), st_));
            NRB_TRY(nrb_approx_bending_energy_gradient(ws_bw_.h, &gbw_, bw(cur_), be_w_, bw(grad_), st_));
        }
        double mf = 0, mb = 0;
        NRB_TRY(nrb_get_maximal_length(fw(grad_), nc_, nullptr, &mf, st_));
        NRB_TRY(nrb_get_maximal_length(bw(grad_), nc_, nullptr, &mb, st_));
        const float mx = std::max((float)mb, (float)mf);
        NRB_TRY(nrb_normalise_gradient(fw(grad_), nc_, (double)mx, nullptr, st_));
        NRB_TRY(nrb_normalise_gradient(bw(grad_), nc_, (double)mx, nullptr, st_));
        return NRB_OK;
    }
    void UpdateBestObjFunctionValue() {
        best_w_measure_ = cur_w_measure_;
        best_w_be_ = cur_w_be_;
        best_nmi_ = cur_nmi_;
        best_be_ = cur_be_;
    }
    nrb_status StoreCurrentDof() {
        NRB_CUDA(cudaMemcpyAsync(best_.p, cur_.p, 6 * nc_ * sizeof(float), cudaMemcpyDeviceToDevice, st_));
        return NRB_OK;
    }
    nrb_status RestoreBestDof() {
        NRB_CUDA(cudaMemcpyAsync(cur_.p, best_.p, 6 * nc_ * sizeof(float), cudaMemcpyDeviceToDevice, st_));
        return NRB_OK;
    }
    // reg_f3d2::UpdateParameters (_reg_f3d2.cpp:652-684): best + scale * gradient for both grids
    // (UpdateVelocityField), then SymmetriseVelocityFields
    nrb_status UpdateParameters(float scale) {
        KernelTimer kt(TK_F2_UPDATE, 0.0, st_);
        NRB_TRY(nrb_update_control_point_position(cur_.p, best_.p, grad_.p, scale, 6 * nc_, st_));
        return symmetrise_velocity(gf_.dim, gfw_.cpp_xyz, fw(cur_), gbw_.cpp_xyz, bw(cur_), st_);
    }
    // ConjugateGradient::Optimise over both grids (reg-lib/Optimiser.cpp:231-323, :129-173)
    nrb_status Optimise(float max_length, float small_length, float& start_length) {
        NRB_TRY(nrb_conjugate_gradient(ws_fw_.h, grad_.p, g1_.p, g2_.p, 6 * nc_, first_call_ ? 1 : 0, st_));
        first_call_ = false;
        size_t line_iteration = 0;
        float added_length = 0;
        float current_length = start_length;
        while (current_length > small_length && line_iteration < 12 && it_ < max_it_) {
            NRB_TRY(UpdateParameters(-current_length));
            double value = 0;
            NRB_TRY(GetObjectiveFunctionValue(true, value));
            if (value > best_obj_) {
                UpdateBestObjFunctionValue();
                best_obj_ = value;
                KeepBestFields();
                added_length += current_length;
                current_length *= 1.1f;
                current_length = std::min(current_length, max_length);
                NRB_TRY(StoreCurrentDof());
            } else {
                current_length *= 0.5;
            }
            ++it_;
            ++line_iteration;
        }
        start_length = added_length;
        return RestoreBestDof();
    }
    // the fields of an accepted trial become the best position's (pointer swaps)
    void KeepBestFields() {
        if (sim_w_ <= 0) return;
        std::swap(def_fw_.p, bdef_fw_.p);
        std::swap(def_bw_.p, bdef_bw_.p);
        std::swap(war_fw_.p, bwar_fw_.p);
        std::swap(war_bw_.p, bwar_bw_.p);
        best_steps_ = steps_;
        best_fields_ = true;
    }
    nrb_status InitLevel(int level, float& max_step);

    nrb_f3d_params p_;
    cudaStream_t st_;
    int levels_ = 0;
    std::vector<Header> hdr_, fhdr_;
    std::vector<DevBuf> ref_pyr_, flo_pyr_;
    Header gf_{}, gb_{};          // forward and backward velocity grids (same dims)
    nrb_geometry gfw_{}, gbw_{};  // reference / floating / forward grid, and swapped / backward grid
    int64_t nc_ = 0;
    int steps_ = 6;               // squaring number (the grids' intent_p2)
    DevBuf ref_, flo_, cur_, best_, grad_, g1_, g2_;  // dof arrays: [forward | backward]
    DevBuf def_fw_, def_bw_, war_fw_, war_bw_, wg_fw_, wg_bw_, vg_fw_, vg_bw_, scr_r_, scr_f_, fields_;
    // the deformation fields and warped images of the best position, when best_fields_
    DevBuf bdef_fw_, bdef_bw_, bwar_fw_, bwar_bw_;
    bool best_fields_ = false;
    int best_steps_ = 6;
    int64_t fields_n_ = 0;
    unsigned *mm_ = nullptr;
    nrb_objective *obj_ = nullptr;    // device: BE forward, BE backward, NMI forward, NMI backward
    nrb_objective *obj_h_ = nullptr;  // pinned host copy
    NmiHandle nmi_fw_, nmi_bw_;
    WsHandle ws_fw_, ws_bw_;
    float pad_ = std::numeric_limits<float>::quiet_NaN();
    float sim_w_ = 1, be_w_ = 0;
    size_t it_ = 0, max_it_ = 0;
    bool first_call_ = true;
    double best_obj_ = 0;
    double cur_w_measure_ = 0, cur_w_be_ = 0, best_w_measure_ = 0, best_w_be_ = 0;
    double cur_nmi_ = 0, cur_be_ = 0, best_nmi_ = 0, best_be_ = 0;
    int64_t n_obj_ = 0, n_grad_ = 0;

public:
    ~F3d2Registration() {
        dev_free(mm_, st_);
        dev_free(obj_, st_);
        if (obj_h_) cudaFreeHost(obj_h_);
    }
};

// reg_f3d2::InitCurrentLevel (_reg_f3d2.cpp:52-102) + InitialiseSimilarity + SetOptimiser
nrb_status F3d2Registration::InitLevel(int level, float& max_step) {
    const Header& r = hdr_[level];
    const Header& f = fhdr_[level];
    max_step = std::max(std::max(std::max(r.pixdim[0], r.pixdim[1]), std::max(f.pixdim[0], f.pixdim[1])),
                        std::max(r.pixdim[2], f.pixdim[2]));
    if (level == 0) {
        be_w_ = be_w_ / powf(16.f, (float)(levels_ - 1));
    } else {
        be_w_ = be_w_ * 16.f;
        const Header nf = refine_header(gf_), nb = refine_header(gb_);
        DevBuf refined;
        NRB_TRY(refined.alloc(6 * nf.n(), st_));
        NRB_TRY(grid_refine(gf_.dim, fw(cur_), nf.dim, refined.p, st_));
        NRB_TRY(grid_refine(gb_.dim, bw(cur_), nb.dim, refined.p + 3 * nf.n(), st_));
        std::swap(cur_.p, refined.p);
        gf_ = nf;
        gb_ = nb;
    }
    nc_ = gf_.n();
    fill_geometry(gfw_, r, f, gf_);
    fill_geometry(gbw_, f, r, gb_);
    std::swap(ref_.p, ref_pyr_[level].p);
    std::swap(flo_.p, flo_pyr_[level].p);
    ref_.st = flo_.st = st_;
    const int64_t nr = r.n(), nfv = f.n();
    NRB_TRY(best_.alloc(6 * nc_, st_));
    NRB_TRY(grad_.alloc(6 * nc_, st_));
    NRB_TRY(g1_.alloc(6 * nc_, st_));
    NRB_TRY(g2_.alloc(6 * nc_, st_));
    NRB_TRY(def_fw_.alloc(3 * nr, st_));
    NRB_TRY(war_fw_.alloc(nr, st_));
    NRB_TRY(bdef_fw_.alloc(3 * nr, st_));
    NRB_TRY(bwar_fw_.alloc(nr, st_));
    NRB_TRY(bdef_bw_.alloc(3 * nfv, st_));
    NRB_TRY(bwar_bw_.alloc(nfv, st_));
    best_fields_ = false;  // the level's initial objective keeps the previous squaring number
    NRB_TRY(wg_fw_.alloc(3 * nr, st_));
    NRB_TRY(vg_fw_.alloc(3 * nr, st_));
    NRB_TRY(scr_r_.alloc(3 * nr, st_));
    NRB_TRY(def_bw_.alloc(3 * nfv, st_));
    NRB_TRY(war_bw_.alloc(nfv, st_));
    NRB_TRY(wg_bw_.alloc(3 * nfv, st_));
    NRB_TRY(vg_bw_.alloc(3 * nfv, st_));
    NRB_TRY(scr_f_.alloc(3 * nfv, st_));
    fields_n_ = 0;
    for (WsHandle *w : { &ws_fw_, &ws_bw_ }) {
        nrb_workspace_destroy(w->h);
        w->h = nullptr;
    }
    NRB_TRY(workspace_create_on(&gfw_, st_, &ws_fw_.h));
    NRB_TRY(workspace_create_on(&gbw_, st_, &ws_bw_.h));
    if (!nmi_fw_.h) NRB_TRY(nmi_create_on(p_.ref_bins + 4, p_.flo_bins + 4, st_, &nmi_fw_.h));
    if (!nmi_bw_.h) NRB_TRY(nmi_create_on(p_.flo_bins + 4, p_.ref_bins + 4, st_, &nmi_bw_.h));
    // reg_nmi::InitialiseMeasure: both images rescaled to [2, bins - 3]
    NRB_TRY(rescale_with(ref_.p, nr, 2.f, (float)(p_.ref_bins + 4) - 3.f, ws_fw_.h->fred, st_));
    NRB_TRY(rescale_with(flo_.p, nfv, 2.f, (float)(p_.flo_bins + 4) - 3.f, ws_fw_.h->fred, st_));
    // Optimiser::Initialise: best = current, objective at the start (no optimiser yet, so the
    // squaring number is not updated: _reg_f3d2.cpp:146-148)
    it_ = 0;
    first_call_ = true;
    NRB_TRY(StoreCurrentDof());
    double v = 0;
    NRB_TRY(GetObjectiveFunctionValue(false, v));
    best_obj_ = v;
    return NRB_OK;
}

nrb_status F3d2Registration::Run(const float *ref, const float *flo, const ImageDesc& rd, const ImageDesc& fd,
                                 float *fw_out, float *bw_out, int64_t cap, float *warped_fw, float *warped_bw,
                                 nrb_f3d_result *res) {
    const auto t0 = std::chrono::steady_clock::now();
    levels_ = p_.levels;
    if (levels_ < 1) return fail(NRB_ERR_INVALID, "registration: levels must be >= 1");
    if (p_.ref_bins < 1 || p_.flo_bins < 1) return fail(NRB_ERR_INVALID, "registration: bins must be >= 1");
    pad_ = p_.padding;
    // reg_f3d2::CheckParameters (_reg_f3d2.cpp:119-141): weights normalised by the penalty sum
    be_w_ = p_.bending_energy;
    const float penalty = be_w_;
    if (penalty >= 1) {
        sim_w_ = 0;
        be_w_ /= penalty;
    } else {
        sim_w_ = 1 - penalty;
    }
    NRB_CUDA(dev_alloc(&mm_, 2 * sizeof(unsigned), st_));
    NRB_CUDA(dev_alloc(&obj_, 4 * sizeof(nrb_objective), st_));
    NRB_CUDA(cudaMemsetAsync(obj_, 0, 4 * sizeof(nrb_objective), st_));
    NRB_CUDA(cudaMallocHost(&obj_h_, 4 * sizeof(nrb_objective)));
    NRB_TRY(build_pyramids(ref, flo, rd, fd, levels_, st_, hdr_, fhdr_, ref_pyr_, flo_pyr_));
    // reg_f3d2::Initialise (_reg_f3d2.cpp:539-610): spacing in voxels of the mean of both images'
    // input spacings, times 2^(levels - 1), grids over the coarsest images
    const Header& rin = hdr_[levels_ - 1];
    const Header& fin = fhdr_[levels_ - 1];
    float spacing[3];
    for (int i = 0; i < 3; ++i) {
        float s = p_.spacing[i];
        if (s != s) s = p_.spacing[0];
        if (s < 0) s *= -(rin.pixdim[i] + fin.pixdim[i]) / 2.f;
        spacing[i] = s * powf(2.f, (float)(levels_ - 1));
    }
    gf_ = symmetric_grid_header(hdr_[0], fhdr_[0], spacing);
    gb_ = gf_;
    nc_ = gf_.n();
    NRB_TRY(cur_.alloc(6 * nc_, st_));
    float cxyz[16];
    gf_.xyz(cxyz);
    NRB_TRY(grid_identity(gf_.dim, cxyz, fw(cur_), st_));
    NRB_TRY(grid_identity(gb_.dim, cxyz, bw(cur_), st_));
    steps_ = 6;
    max_it_ = (size_t)p_.max_iterations;
    max_it_ *= (size_t)std::pow(2, levels_ - 1);
    for (int level = 0; level < levels_; ++level) {
        float max_step = 0;
        NRB_TRY(InitLevel(level, max_step));
        float current_size = max_step;
        const float smallest_size = max_step / 100.0f;
        UpdateBestObjFunctionValue();
        if (p_.verbose)
            printf("[nrb] f3d2 level %d/%d grid %dx%dx%d, initial objective %.6f = (wSIM)%.6f - (wBE)%.6g\n",
                   level + 1, levels_, gf_.dim[0], gf_.dim[1], gf_.dim[2], best_obj_, best_w_measure_, best_w_be_);
        bool just_restarted = false;
        while (current_size) {
            if (it_ >= max_it_) break;
            NRB_TRY(GetObjectiveFunctionGradient());
            current_size = std::min(current_size, max_step);
            NRB_TRY(Optimise(max_step, smallest_size, current_size));
            if (p_.verbose)
                printf("[nrb] [%zu] objective %.6f = (wSIM)%.6f - (wBE)%.6g [+ %g mm], N = %d\n", it_, best_obj_,
                       best_w_measure_, best_w_be_, current_size, steps_);
            if (current_size == 0) {
                if (!just_restarted && it_ < max_it_) {
                    first_call_ = true;
                    current_size = max_step;
                    just_restarted = true;
                }
            } else {
                just_restarted = false;
            }
        }
        max_it_ /= 2;
    }
    const int64_t n = 3 * nc_;
    if ((fw_out || bw_out) && cap < n) return fail(NRB_ERR_INVALID, "registration: grid output capacity too small");
    if (fw_out) NRB_CUDA(cudaMemcpyAsync(fw_out, fw(cur_), n * sizeof(float), cudaMemcpyDefault, st_));
    if (bw_out) NRB_CUDA(cudaMemcpyAsync(bw_out, bw(cur_), n * sizeof(float), cudaMemcpyDefault, st_));
    if (warped_fw || warped_bw) {
        // reg_f3d2::GetWarpedImage (_reg_f3d2.cpp:686-700): the input images through both
        // transformations at full resolution, cubic spline, squaring number as it stands
        const Header& rf = hdr_[levels_ - 1];
        const Header& ff = fhdr_[levels_ - 1];
        nrb_geometry wf{}, wb{};
        fill_geometry(wf, rf, ff, gf_);
        fill_geometry(wb, ff, rf, gb_);
        DevBuf rimg, fimg, def, scr, out;
        NRB_TRY(rimg.alloc(rf.n(), st_));
        NRB_TRY(fimg.alloc(ff.n(), st_));
        NRB_TRY(def.alloc(3 * std::max(rf.n(), ff.n()), st_));
        NRB_TRY(scr.alloc(3 * std::max(rf.n(), ff.n()), st_));
        NRB_TRY(out.alloc(std::max(rf.n(), ff.n()), st_));
        NRB_CUDA(cudaMemcpyAsync(rimg.p, ref, rf.n() * sizeof(float), cudaMemcpyDefault, st_));
        NRB_CUDA(cudaMemcpyAsync(fimg.p, flo, ff.n() * sizeof(float), cudaMemcpyDefault, st_));
        int N = steps_;
        if (warped_fw) {
            NRB_TRY(velocity_to_deformation(&wf, fw(cur_), false, &N, def.p, nullptr, scr.p, mm_, st_));
            NRB_TRY(nrb_resample_image_order(&wf, fimg.p, def.p, nullptr, 3, pad_, out.p, st_));
            NRB_CUDA(cudaMemcpyAsync(warped_fw, out.p, rf.n() * sizeof(float), cudaMemcpyDefault, st_));
        }
        if (warped_bw) {
            NRB_TRY(velocity_to_deformation(&wb, bw(cur_), false, &N, def.p, nullptr, scr.p, mm_, st_));
            NRB_TRY(nrb_resample_image_order(&wb, rimg.p, def.p, nullptr, 3, pad_, out.p, st_));
            NRB_CUDA(cudaMemcpyAsync(warped_bw, out.p, ff.n() * sizeof(float), cudaMemcpyDefault, st_));
        }
        NRB_CUDA(cudaStreamSynchronize(st_));
    }
    NRB_CUDA(cudaStreamSynchronize(st_));
    if (res) {
        for (int i = 0; i < 3; ++i) res->cpp_dim[i] = gf_.dim[i];
        res->final_nmi = best_nmi_;
        res->final_be = best_be_;
        res->final_objective = best_obj_;
        res->objective_evaluations = n_obj_;
        res->gradient_evaluations = n_grad_;
        res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    return NRB_OK;
}

}  // namespace
}  // namespace nrb

// The finest level's velocity grid of a registration, from the image headers alone: the
// symmetric grid over the coarsest pyramid images (reg_f3d2::Initialise, _reg_f3d2.cpp:539-566),
// refined once per finer level (reg_spline_refineControlPointGrid without a reference image).
// F3d2Registration::Run builds the same sequence on the device.
static Header final_velocity_grid(const ImageDesc& rd, const ImageDesc& fd, const nrb_f3d_params *p) {
    const int levels = std::max(1, (int)p->levels);
    std::vector<Header> hdr(levels), fhdr(levels);
    hdr[levels - 1] = header_of(rd);
    fhdr[levels - 1] = header_of(fd);
    for (int l = levels - 2; l >= 0; --l) {
        hdr[l] = halve(hdr[l + 1]);
        fhdr[l] = halve(fhdr[l + 1]);
    }
    float spacing[3];
    for (int i = 0; i < 3; ++i) {
        float sp = p->spacing[i];
        if (sp != sp) sp = p->spacing[0];
        if (sp < 0) sp *= -(hdr[levels - 1].pixdim[i] + fhdr[levels - 1].pixdim[i]) / 2.f;
        spacing[i] = sp * powf(2.f, (float)(levels - 1));
    }
    Header g = symmetric_grid_header(hdr[0], fhdr[0], spacing);
    for (int l = 1; l < levels; ++l) g = refine_header(g);
    return g;
}

static void image_desc(const nrb_image *img, ImageDesc& d) {
    for (int i = 0; i < 3; ++i) {
        d.dim[i] = img->dim[i];
        d.pixdim[i] = img->pixdim[i];
    }
    d.xyz = img->xyz;
    d.sform = img->sform_code > 0;
}

extern "C" nrb_status nrb_f3d2_grid_header(const nrb_image *ref, const nrb_image *flo, const nrb_f3d_params *p,
                                           int32_t dim_out[3], float pixdim_out[3], float xyz_out[16]) {
    if (!ref || !flo || !p || !dim_out || !pixdim_out || !xyz_out)
        return fail(NRB_ERR_INVALID, "nrb_f3d2_grid_header: null pointer");
    for (const nrb_image *img : { ref, flo })
        for (int i = 0; i < 3; ++i)
            if (img->dim[i] < 2 || !(img->pixdim[i] > 0))
                return fail(NRB_ERR_INVALID, "nrb_f3d2_grid_header: 3D images with positive voxel sizes expected");
    ImageDesc rd, fd;
    image_desc(ref, rd);
    image_desc(flo, fd);
    const Header g = final_velocity_grid(rd, fd, p);
    for (int i = 0; i < 3; ++i) {
        dim_out[i] = g.dim[i];
        pixdim_out[i] = g.pixdim[i];
    }
    g.xyz(xyz_out);
    return NRB_OK;
}

// The finest level's control-point grid of an F3D registration from the reference's header: the
// grid of reg_createControlPointGrid over the coarsest reference (spacing x 2^(levels - 1)), then
// reg_spline_refineControlPointGrid onto each finer reference, as F3dRegistration::CreateGrid and
// InitLevel build it on the device.
static Header final_control_grid(const ImageDesc& rd, const nrb_f3d_params *p) {
    const int levels = std::max(1, (int)p->levels);
    std::vector<Header> hdr(levels);
    hdr[levels - 1] = header_of(rd);
    for (int l = levels - 2; l >= 0; --l) hdr[l] = halve(hdr[l + 1]);
    float spacing[3];
    for (int i = 0; i < 3; ++i) {
        float sp = p->spacing[i];
        if (sp != sp) sp = p->spacing[0];
        const float mm = sp < 0 ? sp * -hdr[levels - 1].pixdim[i] : sp;
        spacing[i] = mm * powf(2.f, (float)(levels - 1));
    }
    Header g = grid_header(hdr[0], spacing);
    for (int l = 1; l < levels; ++l) {
        const float half[3] = { g.pixdim[0] / 2.0f, g.pixdim[1] / 2.0f, g.pixdim[2] / 2.0f };
        g = grid_header(hdr[l], half);
    }
    return g;
}

extern "C" nrb_status nrb_f3d_grid_header(const nrb_image *ref, const nrb_f3d_params *p, int32_t dim_out[3],
                                          float pixdim_out[3], float xyz_out[16]) {
    if (!ref || !p || !dim_out || !pixdim_out || !xyz_out) return fail(NRB_ERR_INVALID, "nrb_f3d_grid_header: null pointer");
    for (int i = 0; i < 3; ++i)
        if (ref->dim[i] < 2 || !(ref->pixdim[i] > 0))
            return fail(NRB_ERR_INVALID, "nrb_f3d_grid_header: a 3D image with positive voxel sizes expected");
    ImageDesc rd;
    image_desc(ref, rd);
    const Header g = final_control_grid(rd, p);
    for (int i = 0; i < 3; ++i) {
        dim_out[i] = g.dim[i];
        pixdim_out[i] = g.pixdim[i];
    }
    g.xyz(xyz_out);
    return NRB_OK;
}

// reg_createImagePyramid<float> (reg-lib/cpu/_reg_tools.cpp:1705-1733) of one device image: the
// headers on the host (halve), every coarser level smoothed and downsampled on the device from
// the next finer one, the levels laid end to end in `out`, coarsest first.
extern "C" nrb_status nrb_image_pyramid(const float *img, const int32_t dim[3], const float pixdim[3],
                                        const float xyz[16], int levels, float *out, int64_t capacity,
                                        int32_t *dims_out, float *xyz_out, int64_t *total_out, void *stream) {
    if (!dim || !pixdim || levels < 1 || levels > 16)
        return fail(NRB_ERR_INVALID, "nrb_image_pyramid: dims, spacings and 1..16 levels expected");
    for (int i = 0; i < 3; ++i)
        if (dim[i] < 1 || !(pixdim[i] > 0) || !std::isfinite(pixdim[i]))
            return fail(NRB_ERR_INVALID, "nrb_image_pyramid: positive dims and voxel sizes expected");
    ImageDesc d;
    for (int i = 0; i < 3; ++i) {
        d.dim[i] = dim[i];
        d.pixdim[i] = pixdim[i];
    }
    d.xyz = xyz;
    d.sform = xyz != nullptr;
    std::vector<Header> h(levels);
    h[levels - 1] = header_of(d);
    for (int l = levels - 2; l >= 0; --l) h[l] = halve(h[l + 1]);
    std::vector<int64_t> off(levels + 1, 0);
    for (int l = 0; l < levels; ++l) {
        off[l + 1] = off[l] + h[l].n();
        if (dims_out) memcpy(dims_out + 3 * l, h[l].dim, 3 * sizeof(int32_t));
        if (xyz_out) h[l].xyz(xyz_out + 16 * l);
    }
    if (total_out) *total_out = off[levels];
    if (!out) return NRB_OK;  // headers only
    if (!img) return fail(NRB_ERR_INVALID, "nrb_image_pyramid: null image");
    if (capacity < off[levels]) return fail(NRB_ERR_INVALID, "nrb_image_pyramid: output capacity below the total");
    cudaStream_t st = as_stream(stream);
    NRB_CUDA(cudaMemcpyAsync(out + off[levels - 1], img, h[levels - 1].n() * sizeof(float), cudaMemcpyDeviceToDevice,
                             st));
    if (levels == 1) return NRB_OK;
    DevBuf tmp;
    NRB_TRY(tmp.alloc(4 * h[levels - 1].n(), st));
    for (int l = levels - 2; l >= 0; --l) {
        float nxyz[16], oijk[16];
        h[l].xyz(nxyz);
        h[l + 1].ijk(oijk);
        NRB_TRY(smooth_and_downsample(out + off[l + 1], h[l + 1].dim, out + off[l], h[l].dim, nxyz, oijk, tmp.p, st));
    }
    return NRB_OK;  // tmp is freed in stream order
}

// reg_spline_refineControlPointGrid3D's node values (reg-lib/cpu/_reg_localTrans.cpp:1930-2119):
// the grid of old_dim nodes refined onto new_dim nodes at half the spacing, three planes each
extern "C" nrb_status nrb_refine_control_point_grid(const float *old, const int32_t old_dim[3], float *out,
                                                    const int32_t new_dim[3], void *stream) {
    if (!old || !old_dim || !out || !new_dim) return fail(NRB_ERR_INVALID, "nrb_refine_control_point_grid: null pointer");
    for (int i = 0; i < 3; ++i)
        if (old_dim[i] < 1 || new_dim[i] < 1 || new_dim[i] > 2 * old_dim[i])
            return fail(NRB_ERR_INVALID, "nrb_refine_control_point_grid: new dims must be in [1, 2 * old dims]");
    if (old == out) return fail(NRB_ERR_INVALID, "nrb_refine_control_point_grid: the output aliases the input");
    return grid_refine(old_dim, old, new_dim, out, as_stream(stream));
}

// a velocity grid as NiftyReg tags one (reg_f3d2::Initialise, _reg_f3d2.cpp:596-599)
static void velocity_grid_image(const Header& g, int steps, float *data, nrb_image *out) {
    for (int i = 0; i < 3; ++i) {
        out->dim[i] = g.dim[i];
        out->pixdim[i] = g.pixdim[i];
    }
    out->nvol = 3;
    g.xyz(out->xyz);
    g.ijk(out->ijk);
    out->sform_code = 1;
    out->qform_code = 0;
    out->intent_code = 1007;  // NIFTI_INTENT_VECTOR
    out->intent_p1 = 6.f;     // SPLINE_VEL_GRID
    out->intent_p2 = (float)steps;
    strncpy(out->intent_name, "NREG_TRANS", sizeof(out->intent_name) - 1);
    out->data = data;
}

extern "C" nrb_status nrb_f3d2_register_images(const nrb_image *ref, const nrb_image *flo, const nrb_f3d_params *p,
                                               nrb_image *cpp_fw_out, nrb_image *cpp_bw_out, nrb_image *warped_fw_out,
                                               nrb_image *warped_bw_out, nrb_f3d_result *result) {
    NRB_TRY(check_image(ref, "reference"));
    NRB_TRY(check_image(flo, "floating"));
    if (!p || !cpp_fw_out || !cpp_bw_out) return fail(NRB_ERR_INVALID, "nrb_f3d2_register_images: null pointer");
    for (nrb_image *o : { cpp_fw_out, cpp_bw_out, warped_fw_out, warped_bw_out })
        if (o) memset(o, 0, sizeof(*o));
    ImageDesc rd, fd;
    for (int i = 0; i < 3; ++i) {
        rd.dim[i] = ref->dim[i];
        rd.pixdim[i] = ref->pixdim[i];
        fd.dim[i] = flo->dim[i];
        fd.pixdim[i] = flo->pixdim[i];
    }
    rd.xyz = ref->xyz;
    rd.sform = ref->sform_code > 0;
    fd.xyz = flo->xyz;
    fd.sform = flo->sform_code > 0;
    const int64_t nref = (int64_t)ref->dim[0] * ref->dim[1] * ref->dim[2];
    const int64_t nflo = (int64_t)flo->dim[0] * flo->dim[1] * flo->dim[2];
    const auto t0 = std::chrono::steady_clock::now();
    cudaStream_t st = nullptr;
    NRB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    // the buffers a level or an evaluation frees stay in the pool for the next. Per voxel of
    // the larger image at the finest level, both directions: deformation, warped, image and voxel
    // gradients, scratch (52 B), the best position's deformation and warped image (16 B), the
    // intermediate fields (12 B per squaring, up to 16 kept here), the pyramids, and slack.
    {
        const int64_t big = std::max(nref, nflo);
        keep_pool(big * (2 * 52 + 2 * 16 + 16 * 12 + 2 * 8 * 2) + (256LL << 20));
    }
    nrb_status s = NRB_OK;
    float *fw = nullptr, *bw = nullptr, *wf = nullptr, *wb = nullptr;
    {
        F3d2Registration reg(*p, st);
        // the final grid's size from the headers alone (the registration builds the same), so
        // that the results go straight into host buffers
        const Header g = final_velocity_grid(rd, fd, p);
        const int64_t ncpp = 3 * g.n();
        fw = (float *)malloc((size_t)ncpp * sizeof(float));
        bw = (float *)malloc((size_t)ncpp * sizeof(float));
        wf = warped_fw_out ? (float *)malloc((size_t)nref * sizeof(float)) : nullptr;
        wb = warped_bw_out ? (float *)malloc((size_t)nflo * sizeof(float)) : nullptr;
        if (!fw || !bw || (warped_fw_out && !wf) || (warped_bw_out && !wb)) {
            s = fail(NRB_ERR_OOM, "nrb_f3d2_register_images: host allocation failed");
        } else {
            s = reg.Run(ref->data, flo->data, rd, fd, fw, bw, ncpp, wf, wb, result);
        }
        if (s == NRB_OK) {
            velocity_grid_image(reg.grid_fw(), reg.steps(), fw, cpp_fw_out);
            velocity_grid_image(reg.grid_bw(), reg.steps(), bw, cpp_bw_out);
        }
    }
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (s != NRB_OK) {
        free(fw);
        free(bw);
        free(wf);
        free(wb);
        return s;
    }
    if (warped_fw_out) {
        for (int i = 0; i < 3; ++i) {
            warped_fw_out->dim[i] = ref->dim[i];
            warped_fw_out->pixdim[i] = ref->pixdim[i];
        }
        warped_fw_out->nvol = 1;
        memcpy(warped_fw_out->xyz, ref->xyz, sizeof(ref->xyz));
        memcpy(warped_fw_out->ijk, ref->ijk, sizeof(ref->ijk));
        warped_fw_out->sform_code = ref->sform_code;
        warped_fw_out->qform_code = ref->qform_code;
        warped_fw_out->data = wf;
    }
    if (warped_bw_out) {
        for (int i = 0; i < 3; ++i) {
            warped_bw_out->dim[i] = flo->dim[i];
            warped_bw_out->pixdim[i] = flo->pixdim[i];
        }
        warped_bw_out->nvol = 1;
        memcpy(warped_bw_out->xyz, flo->xyz, sizeof(flo->xyz));
        memcpy(warped_bw_out->ijk, flo->ijk, sizeof(flo->ijk));
        warped_bw_out->sform_code = flo->sform_code;
        warped_bw_out->qform_code = flo->qform_code;
        warped_bw_out->data = wb;
    }
    if (result) result->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return NRB_OK;
}

// reg-apps/reg_f3d.cpp:652-700: the backward result's name inserts "_backward" before the
// .nii.gz / .nii extension (else appends "_backward.nii")
static std::string backward_name(const std::string& f) {
    for (const char *ext : { ".nii.gz", ".nii" }) {
        const size_t at = f.find(ext);
        if (at != std::string::npos) return f.substr(0, at) + "_backward" + ext + f.substr(at + strlen(ext));
    }
    return f + "_backward.nii";
}

extern "C" nrb_status nrb_f3d2_register_files(const char *ref_path, const char *flo_path, const nrb_f3d_params *p,
                                              const char *cpp_path, const char *res_path, nrb_f3d_result *result) {
    if (!ref_path || !flo_path || !p || !cpp_path) return fail(NRB_ERR_INVALID, "nrb_f3d2_register_files: null pointer");
    nrb_image ref{}, flo{}, cf{}, cb{}, wf{}, wb{};
    nrb_status s = nrb_image_read(ref_path, &ref);
    if (s == NRB_OK) s = nrb_image_read(flo_path, &flo);
    if (s == NRB_OK)
        s = nrb_f3d2_register_images(&ref, &flo, p, &cf, &cb, res_path ? &wf : nullptr, res_path ? &wb : nullptr,
                                     result);
    if (s == NRB_OK) s = nrb_image_write(cpp_path, &cf);
    if (s == NRB_OK) s = nrb_image_write(backward_name(cpp_path).c_str(), &cb);
    if (s == NRB_OK && res_path) s = nrb_image_write(res_path, &wf);
    if (s == NRB_OK && res_path) s = nrb_image_write(backward_name(res_path).c_str(), &wb);
    for (nrb_image *img : { &ref, &flo, &cf, &cb, &wf, &wb }) nrb_image_free(img);
    return s;
}
