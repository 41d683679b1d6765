// Device-side state objects behind the opaque handles of the C ABI.
#pragma once

#include <vector>

#include "nrb_common.cuh"

// Fixed number of partial sums every reduction in this library produces before its final
// fixed-order pass; it bounds the grid of the reduction kernels so results never depend on the
// device's SM count.
constexpr int NRB_RED_BLOCKS = 512;
constexpr int NRB_RED_THREADS = 256;

namespace nrb {

// Work decomposition of the voxel passes: an item is a column of 32 x ty voxels over a chunk of
// `zchunk` slices; a block of ty warps stages the item's control points once and each thread
// walks its voxel column along z. The objective pass uses tall blocks (one shared histogram for
// 16 warps leaves most of the SM's L1 to the floating-image gathers); the gradient pass, whose
// threads carry more registers, uses 4 warps.
constexpr int COL_X = 32;
constexpr int TY_OBJECTIVE = 16, TY_GRADIENT = 4, TY_DEFORMATION = 4;

// A floating image (with its margin) held as a 2D layered float array, one layer per z slice,
// and its texture object. Arrays are pooled per process and reused across registrations:
// allocating and freeing them is not ordered on a stream, so the pool keeps that out of the
// registrations' paths (up to a cap on the bytes it keeps unused).
struct FloTexture {
    cudaArray_t arr = nullptr;
    unsigned long long tex = 0;
    int width = 0, height = 0, layers = 0, device = -1;
};
nrb_status flo_texture_acquire(int width, int height, int layers, FloTexture& out);
void flo_texture_release(FloTexture& t);
// copies a dense [layers][height][width] volume into the array's corner, on `st`
nrb_status flo_texture_upload(const FloTexture& t, const float *src, int width, int height, int layers,
                              cudaStream_t st);

// Launch-time description of one voxel walk (a pair's reference volume, grid and floating image,
// and the walk plan's item decomposition).
struct WalkParams {
    int nx, ny, nz;          // reference / deformation-field dims
    int cx, cy, cz;          // control-point grid dims
    float gsx, gsy, gsz;     // grid spacing in reference voxels (grid pixdim / ref pixdim)
    int ty, tiles_x, tiles_y, zchunk, nitems;
    int sa, sb, sc;          // shared strides of the staged block (max spans)
    int fnx, fny, fnz;       // floating dims
    int fsy, fsz, fmargin;   // floating layout: row and slice strides, margin (sample_floating)
    unsigned long long ftex; // the floating image with its margin as a layered texture (0: none)
    Mat34 flo_ijk;           // mm -> floating voxel
    int flo_diag;            // flo_ijk has no off-diagonal terms
    float pad;               // padding value of out-of-volume taps
    int rb, fb;              // internal bin counts
    int cnv;                 // control points per component
    int log_in_smem;         // gradient: an FP32 copy of the log table is staged in shared memory
    int xs;                  // objective: x-contracted rows of the item staged in shared memory
    // identity split of the positions (grid matrix without off-diagonal terms; zero otherwise):
    // node k of axis c sits at io[c] + is[c] * k mm when the transformation is the identity
    float io[3], is[3];
};

// State of the device-resident optimiser (ConjugateGradient::Optimise and the level loop of
// reg_base::Run) that the control kernels of a level's CUDA graph advance.
struct OptState {
    double best_obj, best_w_measure, best_w_be, best_nmi, best_be;
    long long it, max_it, n_obj, n_grad;
    float current_size, max_step, small_step;
    float cur_len;   // step length of the next line-search evaluation
    float step_len;  // step length of the last evaluation (applied to `best` when accepted)
    float added_len;
    int line_iter, first_call, just_restarted, accepted;
    int best_buf;    // NMI table set (0: pro/logt/last, 1: pro2/logt2/last2) of the best position
    int phase;       // batched levels: what the pair needs next (BatchPhase)
};

// Loop conditions of reg_base::Run's level loop and Optimiser::Optimise's line search
// (reg-lib/_reg_base.cpp:760-794, reg-lib/Optimiser.cpp:140-168).
__device__ __forceinline__ bool outer_continues(const OptState& s) { return s.current_size != 0.f && s.it < s.max_it; }
__device__ __forceinline__ bool line_continues(const OptState& s) {
    return s.cur_len > s.small_step && s.line_iter < 12 && s.it < s.max_it;
}

// End of Optimise (start length = added length) and the restart rule of _reg_base.cpp:784-793;
// returns whether the level goes on
__device__ __forceinline__ bool line_end(OptState *s) {
    s->current_size = s->added_len;
    if (s->current_size == 0.f) {
        if (!s->just_restarted && s->it < s->max_it) {
            s->first_call = 1;
            s->current_size = s->max_step;
            s->just_restarted = 1;
        }
    } else {
        s->just_restarted = 0;
    }
    return outer_continues(*s);
}

// Start of Optimise after a gradient evaluation: iteration counted, current_size =
// min(current_size, max_step), first_call consumed, line search set up; returns whether the line
// search runs at all
__device__ __forceinline__ bool gradient_done_line_start(OptState *s) {
    s->it += 1;
    s->n_grad += 1;
    s->current_size = s->max_step < s->current_size ? s->max_step : s->current_size;
    s->first_call = 0;
    s->line_iter = 0;
    s->added_len = 0.f;
    s->cur_len = s->current_size;
    return line_continues(*s);
}

// ---------------------------------------------------------------------------------------------
// Batched levels: many registrations advanced together, one launch per stage over every pair
// that needs that stage. A pair's phase says what it needs next.
// ---------------------------------------------------------------------------------------------
enum BatchPhase : int {
    PH_DONE = 0,  // the level is over for this pair
    PH_INIT = 1,  // the objective at the level's starting point (ConjugateGradient::Initialise)
    PH_LINE = 2,  // a line-search step: the objective at best - cur_len * grad
    PH_GRAD = 3,  // a gradient evaluation at best, then the conjugate-gradient direction
};

// Everything the batched kernels need of one pair at the current level (device array, one per
// pair). Pointers are the pair's own buffers; walks and tables are those its plain
// registration would use, so each pair's arithmetic is the same whatever else is in the batch.
struct BatchPair {
    WalkParams wo, wg;               // objective and gradient walks
    const float *ref, *flo;          // rescaled reference; floating voxel (0, 0, 0) (margin in wo/wg)
    float *best, *grad, *g1, *g2, *vgrad;
    uint32_t *hist;                  // joint counts (zero between evaluations)
    double *pro0, *logt0, *pro1, *logt1;
    nrb_objective *last0, *last1, *obj;
    int rb, fb;
    double *be_partials;
    int n_be;                        // bending-energy partials (blocks of the plain k_be_value)
    double be_norm;                  // 3 * nodes
    float *be_der;                   // 18 derivative values per node
    float be_ratio;                  // bending-energy weight / nodes
    Mat34 grid_xyz;                  // node -> mm (identity positions of k_be_derivatives)
    int rdim[3], cdim[3];
    long long nnode;
    double *red;                     // node-tail partials (2 * NRB_RED_BLOCKS doubles)
    // convolution to the nodes (the aligned-grid passes of launch_convolve_to_nodes)
    int ns[3], radius[3];
    const int *samples[3], *tap_slot[3];
    const float *tap_weight[3], *kernel[3];
    float *conv1, *conv2;
    float node_weight;               // similarity weight x grid/voxel spacing ratios
    Mat34 flo_ijk;                   // reorientation of the node gradient
    double sim_w, be_w;
    OptState *st;
    int obj_items, grad_items, xblocks;
};

constexpr int BATCH_MAX_PAIRS = 64;

// Per-pair tables of the batched voxel passes, passed whole as __grid_constant__ kernel
// parameters: a pair's walk and pointers are then read with uniform constant-bank loads, with no
// copy into shared memory and nothing held in registers.
struct BatchObjEntry {
    WalkParams P;
    const float *ref, *flo, *best, *grad;
    uint32_t *hist;
};
struct BatchObjTable {
    BatchObjEntry e[BATCH_MAX_PAIRS];
};
struct BatchGradEntry {
    WalkParams P;
    const float *ref, *flo, *best;
    float *vgrad;
    const double *logt0, *logt1;
    const nrb_objective *last0, *last1;
};
struct BatchGradTable {
    BatchGradEntry e[BATCH_MAX_PAIRS];
};

// Launch shapes of a batched level, derived on the host from every pair (shared memory for the
// largest walk, template choices every pair allows), and the voxel passes' tables.
struct BatchLaunch {
    int npairs = 0;
    BatchObjTable obj_table;
    BatchGradTable grad_table;
    bool obj_xs = false, obj_diag = false, grad_f32 = false, grad_diag = false;
    size_t obj_smem = 0, grad_smem = 0, fin_smem = 0;
    int obj_grid = 0, grad_grid = 0;
};

// The pairs a batched stage serves (their phase is in `mask`) with the cost of their work units,
// built by warp 0 of every block from the pairs' device state (each block builds the same list)
// and laid out as cost prefix sums. A block then takes the units whose start cost falls in its
// equal share of the total, in pair order, so each block touches few pairs and the shares are
// balanced when units of different pairs cost differently.
struct BatchList {
    int n;                           // pairs served
    long long total;                 // their summed cost
    int pair[BATCH_MAX_PAIRS];       // pair index
    int units[BATCH_MAX_PAIRS];      // work units of the pair
    int w[BATCH_MAX_PAIRS];          // cost of one unit
    long long pref[BATCH_MAX_PAIRS + 1];
};

template <typename F>
__device__ __forceinline__ void batch_list_build(const OptState *__restrict__ states, int npairs, unsigned mask,
                                                 F units_of, BatchList& L) {
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int n = 0;
        long long total = 0;
        for (int base = 0; base < npairs; base += 32) {
            const int p = base + lane;
            int u = 0, w = 0;
            if (p < npairs && ((mask >> states[p].phase) & 1u)) units_of(p, u, w);
            const long long c = (long long)u * w;
            long long inc = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const long long v = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += v;
            }
            const unsigned act = __ballot_sync(0xffffffffu, u > 0);
            if (u > 0) {
                const int slot = n + __popc(act & ((1u << lane) - 1u));
                L.pair[slot] = p;
                L.units[slot] = u;
                L.w[slot] = w;
                L.pref[slot] = total + inc - c;
            }
            total += __shfl_sync(0xffffffffu, inc, 31);
            n += __popc(act);
        }
        if (lane == 0) {
            L.n = n;
            L.total = total;
            L.pref[n] = total;
        }
    }
    __syncthreads();
}

// A block's share of a batched stage as segments (pair, first unit, end unit), in pair order,
// computed once per block into shared memory so that none of the bookkeeping stays live across
// the walk of a unit.
struct BatchSegments {
    int n;
    int pair[BATCH_MAX_PAIRS], j0[BATCH_MAX_PAIRS], j1[BATCH_MAX_PAIRS];
};

__device__ __forceinline__ bool batch_units(const BatchList& L, int k, long long c0, long long c1, int& j0, int& j1);

// the block's equal share of the list's cost (after batch_list_build; ends with a barrier)
__device__ __forceinline__ void batch_segments(const BatchList& L, BatchSegments& G) {
    if (threadIdx.x == 0) {
        const long long c0 = L.total * blockIdx.x / gridDim.x, c1 = L.total * (blockIdx.x + 1) / gridDim.x;
        int n = 0;
        for (int k = 0; k < L.n; ++k) {
            int j0, j1;
            if (!batch_units(L, k, c0, c1, j0, j1)) continue;
            G.pair[n] = L.pair[k];
            G.j0[n] = j0;
            G.j1[n] = j1;
            ++n;
        }
        G.n = n;
    }
    __syncthreads();
}

// units [j0, j1) of active pair k that start in the cost range [c0, c1)
__device__ __forceinline__ bool batch_units(const BatchList& L, int k, long long c0, long long c1, int& j0, int& j1) {
    const long long a = L.pref[k], b = L.pref[k + 1], w = L.w[k];
    if (b <= c0 || a >= c1) return false;
    j0 = c0 > a ? (int)((c0 - a + w - 1) / w) : 0;
    j1 = (int)min((long long)L.units[k], (c1 - a + w - 1) / w);
    return j0 < j1;
}

__device__ __forceinline__ void copy_words(void *dst, const void *src, int bytes) {
    for (int i = threadIdx.x; i < bytes / 4; i += blockDim.x)
        static_cast<int *>(dst)[i] = static_cast<const int *>(src)[i];
}

// The same list walked element-wise: every element of every served pair, grid-stride per pair
template <typename F>
__device__ __forceinline__ void batch_elements(const BatchList& L, F work) {
    const long long gtid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long gs = (long long)gridDim.x * blockDim.x;
    for (int k = 0; k < L.n; ++k)
        for (long long i = gtid; i < L.units[k]; i += gs) work(L.pair[k], i);
}

// Counts of the pairs' phases, by the block that took the last ticket of a per-pair cluster
// launch; that block sets the graph's conditions for the rest of the iteration.
__device__ __forceinline__ void batch_counts(const OptState *states, int npairs, int& nline, int& ngrad) {
    __shared__ int s_line, s_grad;
    if (threadIdx.x == 0) s_line = s_grad = 0;
    __syncthreads();
    int l = 0, g = 0;
    for (int q = threadIdx.x; q < npairs; q += blockDim.x) {
        const int ph = *reinterpret_cast<const volatile int *>(&states[q].phase);
        l += ph == PH_LINE || ph == PH_INIT;
        g += ph == PH_GRAD;
    }
    if (l) atomicAdd(&s_line, l);
    if (g) atomicAdd(&s_grad, g);
    __syncthreads();
    nline = s_line;
    ngrad = s_grad;
}

// Takes the cluster's ticket (block rank 0 of each cluster, every thread of that block); true
// in the block that took the last one, after which every pair's state is visible.
__device__ __forceinline__ bool batch_last_cluster(unsigned int *ticket, unsigned int nclusters) {
    __shared__ unsigned int s_last;
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(ticket, 1u) == nclusters - 1;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        if (threadIdx.x == 0) *ticket = 0u;
    }
    return s_last != 0;
}

// Tickets of the per-pair cluster kernels: the last cluster to finish sets the graph's
// conditions from every pair's phase.
struct BatchCtl {
    unsigned int ticket_fin, ticket_tail;
    int grad_percent;                // run the gradient stage once this share (%) of the active pairs waits for it
    long long iterations, grad_stages;  // graph iterations and gradient stages run (statistics)
    int run_grad, go_on;             // the last decisions (read by the host when it drives the level)
};

// One line-search step of Optimiser::Optimise (reg-lib/Optimiser.cpp:140-168) after its
// objective evaluation: accept (best values, added length, length x 1.1 capped at max_step) or
// halve the length; the objective is the weighted difference of reg_f3d::GetObjectiveFunctionValue
// (reg-lib/_reg_f3d.cpp:443-462). Returns whether the line search goes on.
__device__ __forceinline__ bool line_step(OptState *s, double nmi, double be, double sim_w, double be_w) {
    const double wm = sim_w > 0 ? sim_w * nmi : 0.0;
    const double wb = be_w > 0 ? be_w * be : 0.0;
    const double value = __dsub_rn(wm, wb);
    s->n_obj += 1;
    s->step_len = s->cur_len;
    if (value > s->best_obj) {
        s->best_w_measure = wm;
        s->best_w_be = wb;
        s->best_nmi = nmi;
        s->best_be = be;
        s->best_obj = value;
        s->added_len = __fadd_rn(s->added_len, s->cur_len);
        const float c = __fmul_rn(s->cur_len, 1.1f);
        s->cur_len = s->max_step < c ? s->max_step : c;
        s->accepted = 1;
        s->best_buf ^= 1;  // the evaluation wrote the other table set
    } else {
        s->cur_len = __fmul_rn(s->cur_len, 0.5f);
        s->accepted = 0;
    }
    s->it += 1;
    s->line_iter += 1;
    return s->cur_len > s->small_step && s->line_iter < 12 && s->it < s->max_it;
}

// Trial control-point value of the line search, best + (-len) * grad, with the float operations
// of UpdateControlPointPosition (reg-lib/Compute.cpp:91-127); without grad, the stored value.
__device__ __forceinline__ float trial_cp(const float *__restrict__ cpp, const float *__restrict__ grad, float scale,
                                          long long i) {
    const float b = __ldg(cpp + i);
    return grad ? __fadd_rn(b, __fmul_rn(scale, __ldg(grad + i))) : b;
}

struct WalkPlan {
    int ty = 0;  // warps per block = voxel rows per item
    int tiles_x = 0, tiles_y = 0, zchunk = 0, nchunks = 0, nitems = 0;
    int sa = 0, sb = 0, sc = 0;  // max control-point span of an item along x, y, z
    int cp_floats = 0;           // shared floats of the staged control-point block
    int resident = 0;            // co-resident blocks of the persistent grid; 0 = occupancy limit
};
WalkPlan plan_walk(const nrb_geometry *g, int ty, long long (*slots_for)(size_t smem), size_t extra_smem,
                   int min_chunk = 8, int overhead = 4);
// Second-derivative stencils of the bending energy at the nodes, in the 27-point (c, b, a) order
// of set_second_order_bspline_basis_values (reg-lib/cpu/_reg_splineBasis.cpp:291-455), rounded to
// 6 decimals as the reference tabulates them.
struct BeBasis {
    float v[6][27];  // xx, yy, zz, xy, yz, xz
};
// One component's share of an interior node's bending-energy term: the squares of its three
// second derivatives and the float sum of its three squared cross derivatives.
struct BeTerms {
    float xx, yy, zz, cross;
};
// Component k of interior node n (of ix * iy * iz interior nodes): its 6 stencil sums over the 27
// points in (c, b, a) order without contraction, then the squares. `full_unroll` keeps all 27
// loads in flight (a thread that evaluates one component); otherwise one c-plane at a time.
template <bool full_unroll>
__device__ __forceinline__ BeTerms be_node_component(int cx, int cy, int cz, int ix, int iy,
                                                     const float *__restrict__ cpp, const BeBasis& B,
                                                     const float *__restrict__ grad, float scale, long long n, int k) {
    const long long nc = (long long)cx * cy * cz;
    const int x = 1 + (int)(n % ix);
    const int y = 1 + (int)((n / ix) % iy);
    const int z = 1 + (int)(n / ((long long)ix * iy));
    auto sq = [](float v) { return __fmul_rn(v, v); };
    float d[6];
#pragma unroll
    for (int t = 0; t < 6; ++t) d[t] = 0.f;
#pragma unroll(full_unroll ? 3 : 1)
    for (int c = -1; c < 2; ++c)
#pragma unroll
        for (int b = -1; b < 2; ++b)
#pragma unroll
            for (int a = -1; a < 2; ++a) {
                const int i = 9 * (c + 1) + 3 * (b + 1) + (a + 1);
                const long long idx = ((long long)(z + c) * cy + y + b) * cx + x + a;
                const float v = trial_cp(cpp, grad, scale, k * nc + idx);
#pragma unroll
                for (int t = 0; t < 6; ++t) d[t] = __fadd_rn(d[t], __fmul_rn(B.v[t][i], v));
            }
    return BeTerms{ sq(d[0]), sq(d[1]), sq(d[2]), __fadd_rn(__fadd_rn(sq(d[3]), sq(d[4])), sq(d[5])) };
}
// Adds component k's terms to the node's sum in the reference expression's order: the first
// three squares of component 0 summed in float, every later term added in double.
__device__ __forceinline__ double be_add_component(double s, const BeTerms& t, int k) {
    if (k == 0) return __dadd_rn((double)__fadd_rn(__fadd_rn(t.xx, t.yy), t.zz), __dmul_rn(2.0, (double)t.cross));
    s = __dadd_rn(s, (double)t.xx);
    s = __dadd_rn(s, (double)t.yy);
    s = __dadd_rn(s, (double)t.zz);
    return __dadd_rn(s, __dmul_rn(2.0, (double)t.cross));
}
// the bending-energy value term of interior node n, one component at a time (only 6 sums live)
__device__ __forceinline__ double be_node_value(int cx, int cy, int cz, int ix, int iy, const float *__restrict__ cpp,
                                                const BeBasis& B, const float *__restrict__ grad, float scale,
                                                long long n) {
    double s = 0.0;
#pragma unroll 1
    for (int k = 0; k < 3; ++k)
        s = be_add_component(s, be_node_component<false>(cx, cy, cz, ix, iy, cpp, B, grad, scale, n, k), k);
    return s;
}

// The `count` plans of lowest modelled cost (distinct z-chunks), best first.
std::vector<WalkPlan> plan_walk_candidates(const nrb_geometry *g, int ty, long long (*slots_for)(size_t smem),
                                           size_t extra_smem, int min_chunk, int overhead, int count);
// shared bytes beyond the walk that plan_walk assumes for the objective and gradient passes
constexpr size_t OBJ_PLAN_EXTRA = (size_t)68 * 68 * 4, GRAD_PLAN_EXTRA = (size_t)(68 * 68 + 136) * 4;
size_t walk_smem_bytes(const WalkPlan& W);
// co-resident blocks of the persistent voxel passes for a given dynamic shared-memory size
long long objective_slots(size_t smem);
long long gradient_slots(size_t smem);
long long deformation_slots(size_t smem);

}  // namespace nrb

// One NMI measure: histogram counts (kept zero between evaluations), FP64 tables, entropies.
struct nrb_nmi {
    int rb = 0, fb = 0;            // internal bin counts (user bins + 4)
    int total = 0;                 // rb*fb + rb + fb
    uint32_t *hist = nullptr;      // rb*fb joint counts
    double *pro = nullptr;         // total: smoothed, normalised joint | ref marginal | flo marginal
    double *logt = nullptr;        // total: log of pro (0 where pro == 0)
    nrb_objective *last = nullptr; // entropies / NMI of the last evaluation
    // second set of tables: inside a level graph the evaluations alternate between the two so
    // that the tables of the best position survive rejected line-search steps
    double *pro2 = nullptr, *logt2 = nullptr;
    nrb_objective *last2 = nullptr;
    int device = 0;
    cudaStream_t st = nullptr;     // owner's stream for stream-ordered allocation (or none)
};

// Per-axis description of where the node sampling of Compute::VoxelCentricToNodeCentric reads
// the convolved voxel gradient: the sorted distinct voxel indices ("samples") and, per node,
// up to two (sample slot, trilinear weight) taps.
struct AxisSampling {
    int nsamples = 0;
    std::vector<int> samples;       // voxel index of each slot
    std::vector<int> tap_slot;      // 2 per node (-1 = no tap)
    std::vector<float> tap_weight;  // 2 per node
    std::vector<float> kernel;      // cubic kernel taps, 2*radius+1
    int radius = 0;
};

struct nrb_workspace {
    nrb_geometry g{};
    int device = 0;
    nrb::WalkPlan walk_obj, walk_grad;
    // reduction partials (double pairs) and scalars
    double *red = nullptr;          // 2 * NRB_RED_BLOCKS doubles
    double *be_partials = nullptr;  // NRB_RED_BLOCKS doubles
    float *fred = nullptr;          // 2 * NRB_RED_BLOCKS floats (min | max partials)
    // bending-energy gradient: 18 derivative values per node
    float *be_deriv = nullptr;
    // convolution-at-nodes scratch
    AxisSampling ax[3];
    int *d_samples[3] = { nullptr, nullptr, nullptr };
    int *d_tap_slot[3] = { nullptr, nullptr, nullptr };
    float *d_tap_weight[3] = { nullptr, nullptr, nullptr };
    float *d_kernel[3] = { nullptr, nullptr, nullptr };
    float *conv1 = nullptr;         // [3][nz][ny][nsx]
    float *conv2 = nullptr;         // [3][nz][nsy][nsx]
    // a grid not aligned with the reference (F3D2 grids of rotated images): the voxel gradient is
    // convolved whole in `general_vox` ([3][nz][ny][nx]) and sampled node by node
    bool general = false;
    float *general_vox = nullptr;
    // a registration's floating image with its margin as a layered texture (FloTexture), which the
    // fused passes gather from when they sample that padded image (0: none)
    unsigned long long flo_tex = 0;
    size_t bytes = 0;
    cudaStream_t st = nullptr;      // owner's stream for stream-ordered allocation (or none)
    // the node-grid kernels (bending energy) run on a side stream, overlapped with the voxel
    // passes of the same evaluation: fork/join through two events
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};

namespace nrb {

nrb_status workspace_init(nrb_workspace *ws, const nrb_geometry *g);
// creators whose buffers are allocated and freed in the order of `st` (st may be null)
nrb_status workspace_create_on(const nrb_geometry *g, cudaStream_t st, nrb_workspace **out);
nrb_status nmi_create_on(int ref_bins, int flo_bins, cudaStream_t st, nrb_nmi **out);
void workspace_free(nrb_workspace *ws);
nrb_status validate_geometry(const nrb_geometry *g);

// launchers shared between translation units
// ctl (optional, inside a level graph): the finalize writes the table set that does not hold the
// best position, takes the line-search step and sets the line search's WHILE condition `line`;
// with acc_n > 0 it also stores an accepted trial position: acc_best += -step_len * acc_grad
nrb_status launch_nmi_finalize(nrb_nmi *nmi, const double *be_partials, int n_be_partials,
                               int64_t cpp_nvox3, double sim_weight, double be_weight,
                               nrb_objective *obj, cudaStream_t st, OptState *ctl = nullptr,
                               cudaGraphConditionalHandle line = 0, float *acc_best = nullptr,
                               const float *acc_grad = nullptr, long long acc_n = 0);
// grad/step (optional): evaluate at the line search's trial position cpp - step->cur_len * grad
// flo_margin > 0: `flo` is the voxel (0, 0, 0) of a copy made by pad_volume with that margin
// Walk autotuner: the level's objective and gradient walks (items per block row ty, z-chunk,
// resident blocks) timed on the device over a candidate set, the fastest kept in a process-wide
// table keyed by the level's shape (reference and grid dims, grid spacing in voxels, bins, mask,
// floating margin, texture). The walk plan changes which block visits which voxels, never a
// value: the histogram counts are integers and every other output is per voxel or per node, so
// results are bit-identical whatever the table holds. autotune_walks times the candidates the
// first time a shape is seen (the tables of nmi must hold an evaluation: the gradient pass reads
// them) and leaves the histogram counts zero; later levels of that shape reuse the entry.
// autotune_lookup applies an entry if one exists; with `batched` it applies the best plan among
// those with the batched kernels' block shapes (ty = TY_OBJECTIVE / TY_GRADIENT).
nrb_status autotune_walks(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g, const float *ref, const float *flo,
                          const int32_t *mask, const float *cpp, float padding, int flo_margin, float *vgrad,
                          cudaStream_t st);
bool autotune_lookup(nrb_workspace *ws, const nrb_nmi *nmi, const int32_t *mask, int flo_margin, bool batched);

nrb_status launch_fused_objective(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g,
                                  const float *ref, const float *flo, const int32_t *mask,
                                  const float *cpp, float padding, cudaStream_t st,
                                  const float *grad = nullptr, const OptState *step = nullptr,
                                  int flo_margin = 0);
// sel (optional, inside a level graph): read the NMI table set sel->best_buf
nrb_status launch_fused_gradient(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g,
                                 const float *ref, const float *flo, const int32_t *mask,
                                 const float *cpp, float padding, double weight, float *vgrad,
                                 cudaStream_t st, const OptState *sel = nullptr, int flo_margin = 0);
// Copy of a dense [nz][ny][nx] volume with `margin` voxels of `value` added on every side
// (dst: (nx + 2m) (ny + 2m) (nz + 2m) floats); returns in *origin the copy's voxel (0, 0, 0).
nrb_status pad_volume(const float *src, const int32_t dim[3], int margin, float value, float *dst,
                      const float **origin, cudaStream_t st);
inline long long padded_voxels(const int32_t dim[3], int margin) {
    return (long long)(dim[0] + 2 * margin) * (dim[1] + 2 * margin) * (dim[2] + 2 * margin);
}
// the fused evaluations of nrb_f3d_objective / nrb_f3d_gradient on a floating image laid out
// with `flo_margin` (0: the dense volume of the public entry points)
nrb_status f3d_objective(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g, const float *ref,
                         const float *flo, int flo_margin, const int32_t *mask, const float *cpp, float padding,
                         double sim_weight, double be_weight, nrb_objective *obj, nrb_objective *obj_host,
                         cudaStream_t st);
nrb_status f3d_gradient(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g, const float *ref,
                        const float *flo, int flo_margin, const int32_t *mask, const float *cpp, float padding,
                        double sim_weight, double be_weight, float *vgrad, float *node_grad, cudaStream_t st);
nrb_status launch_be_value(nrb_workspace *ws, const nrb_geometry *g, const float *cpp,
                           cudaStream_t st, const float *grad = nullptr, const OptState *step = nullptr);
nrb_status launch_be_derivatives(nrb_workspace *ws, const nrb_geometry *g, const float *cpp, cudaStream_t st);
nrb_status launch_be_accumulate(nrb_workspace *ws, const nrb_geometry *g, float weight, float *node_grad,
                                cudaStream_t st);
int be_partial_count(const nrb_geometry *g);
// batched levels (csrc/nrb_tile.cu): a pair's walks as its plain registration would launch them
nrb_status batch_walks(nrb_workspace *ws, const nrb_nmi *nmi, const nrb_geometry *g, float padding, int flo_margin,
                       WalkParams& wo, WalkParams& wg);
nrb_status batch_plan(std::vector<BatchPair>& pairs, BatchLaunch& L);
// (bytes: the algorithmic bytes of the launch, for the per-kernel timers when they are on)
nrb_status launch_batch_objective(const BatchPair *d_pairs, const OptState *states, const BatchLaunch& L,
                                  cudaStream_t st, double bytes = 0.0);
nrb_status launch_batch_gradient(const BatchPair *d_pairs, const OptState *states, const BatchLaunch& L,
                                 cudaStream_t st, double bytes = 0.0);
// in_graph: set the level graph's conditions (else the decisions are only left in bctl)
nrb_status launch_batch_finalize(const BatchPair *d_pairs, OptState *states, BatchCtl *bctl, const BatchLaunch& L,
                                 bool in_graph, cudaGraphConditionalHandle grad_if, cudaGraphConditionalHandle outer,
                                 cudaStream_t st);
// batched levels (csrc/nrb_ops.cu): a pair's node-stage description from its workspace, the
// bending-energy value partials of the pairs in INIT / LINE, and the gradient stage of the pairs in
// GRAD around the voxel pass `gradient` (bending-energy derivatives on `side`, the node
// convolution, the bending-energy gradient)
nrb_status batch_node_stage(const nrb_workspace *ws, const nrb_geometry *g, float sim_weight, float be_weight,
                            BatchPair& b);
nrb_status launch_batch_be_value(const std::vector<BatchPair>& hp, const BatchPair *d, const OptState *states,
                                 cudaStream_t st);
nrb_status launch_batch_node_stage(const std::vector<BatchPair>& hp, const BatchPair *d, const OptState *states,
                                   cudaStream_t st, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join,
                                   nrb_status (*gradient)(const BatchPair *, const OptState *, cudaStream_t, void *),
                                   void *gradient_arg);
// batched registrations (csrc/nrb_f3d.cu): n pairs advanced together level by level on `st`
// the NMI voxel gradient (nrb_nmi_voxel_gradient) with the window's precision chosen: fp64 keeps
// the FP64 window whatever the table size
nrb_status nmi_voxel_gradient(nrb_nmi *nmi, const nrb_geometry *g, const float *ref, const float *warped,
                              const float *warped_grad, const int32_t *mask, double weight, float *vgrad,
                              cudaStream_t st, bool fp64);
nrb_status register_batch_fused(const nrb_pair *pairs, int n, const nrb_f3d_params *p, nrb_f3d_result *results,
                                cudaStream_t st, int grad_percent);
// side stream of `ws` starts after the work queued so far on st / st waits for the side stream
nrb_status fork_side(nrb_workspace *ws, cudaStream_t st);
nrb_status join_side(nrb_workspace *ws, cudaStream_t st);
nrb_status launch_convolve_to_nodes(nrb_workspace *ws, const nrb_geometry *g, const float *vgrad,
                                    float weight, float *node, cudaStream_t st);

}  // namespace nrb
