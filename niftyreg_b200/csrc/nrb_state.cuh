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
};
WalkPlan plan_walk(const nrb_geometry *g, int ty, long long (*slots_for)(size_t smem), size_t extra_smem,
                   int min_chunk = 8, int overhead = 4);
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
// side stream of `ws` starts after the work queued so far on st / st waits for the side stream
nrb_status fork_side(nrb_workspace *ws, cudaStream_t st);
nrb_status join_side(nrb_workspace *ws, cudaStream_t st);
nrb_status launch_convolve_to_nodes(nrb_workspace *ws, const nrb_geometry *g, const float *vgrad,
                                    float weight, float *node, cudaStream_t st);

}  // namespace nrb
