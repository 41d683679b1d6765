// Library-level C ABI: error state, device selection, NMI handles and the fused F3D
// objective / gradient evaluations.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "nrb_state.cuh"

namespace nrb {

static thread_local std::string g_error;
std::atomic<long long> g_launch_count{0};

void set_error(const std::string& msg) { g_error = msg; }

nrb_status fail(nrb_status code, const std::string& msg) {
    g_error = msg;
    return code;
}

nrb_status check_cuda(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return NRB_OK;
    g_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? NRB_ERR_OOM : NRB_ERR_CUDA;
}

int sm_count() {
    static std::mutex mu;
    static std::vector<int> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)cache.size() <= dev) cache.resize(dev + 1, 0);
    if (cache[dev] == 0) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cache[dev] = n > 0 ? n : 148;
    }
    return cache[dev];
}

// ---- the library's memory pool ----------------------------------------------------------------
namespace {
std::mutex g_lib_pool_mu;
std::vector<cudaMemPool_t> g_lib_pools;  // by device; null until created
std::vector<char> g_lib_pool_tried;
}  // namespace

cudaMemPool_t lib_pool() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return lib_pool_of(dev);
}

cudaMemPool_t lib_pool_of(int dev) {
    std::lock_guard<std::mutex> lock(g_lib_pool_mu);
    if ((int)g_lib_pools.size() <= dev) {
        g_lib_pools.resize(dev + 1, nullptr);
        g_lib_pool_tried.resize(dev + 1, 0);
    }
    if (!g_lib_pool_tried[dev]) {
        g_lib_pool_tried[dev] = 1;
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) == cudaSuccess) {
            uint64_t thr = kLibPoolFloor;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
            // no reuse across streams through inserted dependencies: registrations running on
            // their own streams (batch workers, server slots) never wait for one another because
            // the pool handed one of them memory the other freed
            int no = 0;
            cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no);
            g_lib_pools[dev] = pool;
        }
        cudaGetLastError();
    }
    return g_lib_pools[dev];
}

void lib_pool_keep(uint64_t bytes) {
    cudaMemPool_t pool = lib_pool();
    if (!pool) return;
    std::lock_guard<std::mutex> lock(g_lib_pool_mu);
    uint64_t cur = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &cur) == cudaSuccess && cur < bytes)
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &bytes);
    cudaGetLastError();
}

// ---- per-kernel timing ----------------------------------------------------------------------
namespace {
struct Pending {
    cudaEvent_t a, b;
    int k;
    double bytes;
};
std::mutex g_tmu;
bool g_timing = false;
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_pool;
long long g_tlaunch[TK_COUNT] = {};
double g_tms[TK_COUNT] = {}, g_tbytes[TK_COUNT] = {};
const char *g_tnames[TK_COUNT] = { "objective", "gradient", "finalize", "conv", "be_value", "be_gradient",
                                   "f3d2_velocity", "f3d2_compose", "f3d2_gradient_exp", "f3d2_warp", "f3d2_nmi",
                                   "f3d2_voxel_gradient", "f3d2_nodes", "f3d2_be", "f3d2_update" };

cudaEvent_t pooled_event() {
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void resolve_pending() {
    for (const Pending& p : g_pending) {
        float ms = 0;
        if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            g_tlaunch[p.k] += 1;
            g_tms[p.k] += ms;
            g_tbytes[p.k] += p.bytes;
        }
        g_pool.push_back(p.a);
        g_pool.push_back(p.b);
    }
    g_pending.clear();
}
}  // namespace

bool timing_enabled() {
    std::lock_guard<std::mutex> lock(g_tmu);
    return g_timing;
}

KernelTimer::KernelTimer(TimedKernel k, double bytes, cudaStream_t st): k_(k), bytes_(bytes), st_(st) {
    std::lock_guard<std::mutex> lock(g_tmu);
    if (!g_timing) return;
    if (g_pending.size() > 4096) resolve_pending();
    a_ = pooled_event();
    cudaEventRecord(a_, st_);
}

KernelTimer::~KernelTimer() {
    if (!a_) return;
    std::lock_guard<std::mutex> lock(g_tmu);
    cudaEvent_t b = pooled_event();
    cudaEventRecord(b, st_);
    g_pending.push_back({ a_, b, (int)k_, bytes_ });
}



}  // namespace nrb

using namespace nrb;

extern "C" const char *nrb_last_error(void) { return g_error.c_str(); }

extern "C" int64_t nrb_kernel_launch_count(void) { return g_launch_count.load(); }

extern "C" void nrb_timing_enable(int on) {
    std::lock_guard<std::mutex> lock(g_tmu);
    resolve_pending();
    if (on) {
        // events are created here, never between a timed launch's two records
        while (g_pool.size() < 16384) {
            cudaEvent_t e = nullptr;
            if (cudaEventCreate(&e) != cudaSuccess) break;
            g_pool.push_back(e);
        }
        for (int k = 0; k < TK_COUNT; ++k) {
            g_tlaunch[k] = 0;
            g_tms[k] = 0;
            g_tbytes[k] = 0;
        }
    }
    g_timing = on != 0;
}

extern "C" nrb_status nrb_timing_read(const char *kernel, int64_t *launches, double *total_ms,
                                      double *algorithmic_bytes) {
    if (!kernel) return fail(NRB_ERR_INVALID, "nrb_timing_read: null name");
    std::lock_guard<std::mutex> lock(g_tmu);
    resolve_pending();
    for (int k = 0; k < TK_COUNT; ++k) {
        if (strcmp(kernel, g_tnames[k]) != 0) continue;
        if (launches) *launches = g_tlaunch[k];
        if (total_ms) *total_ms = g_tms[k];
        if (algorithmic_bytes) *algorithmic_bytes = g_tbytes[k];
        return NRB_OK;
    }
    return fail(NRB_ERR_INVALID, std::string("nrb_timing_read: unknown kernel ") + kernel);
}

extern "C" nrb_status nrb_set_device(int device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(NRB_ERR_NO_DEVICE, "no CUDA device visible");
    }
    if (device < 0 || device >= n) return fail(NRB_ERR_INVALID, "device index out of range");
    NRB_CUDA(cudaSetDevice(device));
    int major = 0;
    NRB_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    if (major != 10) return fail(NRB_ERR_NO_DEVICE, "device is not compute capability 10.x (sm_100a build)");
    return NRB_OK;
}

extern "C" nrb_status nrb_memory_trim(size_t keep_bytes) {
    cudaMemPool_t pool = lib_pool();
    if (!pool) return NRB_OK;  // no pool of the library on this device: nothing held
    NRB_CUDA(cudaMemPoolTrimTo(pool, keep_bytes));
    return NRB_OK;
}

extern "C" int nrb_device_ok(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return 0;
    }
    int dev = 0, major = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    return major == 10 ? 1 : 0;
}

namespace nrb {
nrb_status nmi_create_on(int ref_bins, int flo_bins, cudaStream_t st, nrb_nmi **out) {
    if (!out || ref_bins < 5 || flo_bins < 5 || ref_bins > 1024 || flo_bins > 1024)
        return fail(NRB_ERR_INVALID, "nrb_nmi_create: bins must be in [5, 1024] (internal counts, user bins + 4)");
    if ((size_t)ref_bins * flo_bins * 4 > 180 * 1024)
        return fail(NRB_ERR_UNSUPPORTED, "nrb_nmi_create: joint histogram larger than one SM's shared memory");
    nrb_nmi *n = new nrb_nmi();
    n->rb = ref_bins;
    n->fb = flo_bins;
    n->total = ref_bins * flo_bins + ref_bins + flo_bins;
    n->st = st;
    cudaGetDevice(&n->device);
    const size_t hb = (size_t)ref_bins * flo_bins * 4, tb = (size_t)n->total * 8;
    bool ok = dev_alloc(&n->hist, hb, st) == cudaSuccess && dev_alloc(&n->pro, tb, st) == cudaSuccess &&
              dev_alloc(&n->logt, tb, st) == cudaSuccess && dev_alloc(&n->last, sizeof(nrb_objective), st) == cudaSuccess &&
              dev_alloc(&n->pro2, tb, st) == cudaSuccess && dev_alloc(&n->logt2, tb, st) == cudaSuccess &&
              dev_alloc(&n->last2, sizeof(nrb_objective), st) == cudaSuccess;
    if (ok && st) {
        ok = cudaMemsetAsync(n->hist, 0, hb, st) == cudaSuccess && cudaMemsetAsync(n->pro, 0, tb, st) == cudaSuccess &&
             cudaMemsetAsync(n->logt, 0, tb, st) == cudaSuccess &&
             cudaMemsetAsync(n->last, 0, sizeof(nrb_objective), st) == cudaSuccess &&
             cudaMemsetAsync(n->last2, 0, sizeof(nrb_objective), st) == cudaSuccess;
    } else if (ok) {
        ok = cudaMemset(n->hist, 0, hb) == cudaSuccess && cudaMemset(n->pro, 0, tb) == cudaSuccess &&
             cudaMemset(n->logt, 0, tb) == cudaSuccess && cudaMemset(n->last, 0, sizeof(nrb_objective)) == cudaSuccess &&
             cudaMemset(n->last2, 0, sizeof(nrb_objective)) == cudaSuccess;
    }
    if (!ok) {
        cudaGetLastError();
        nrb_nmi_destroy(n);
        return fail(NRB_ERR_OOM, "nrb_nmi_create: device allocation failed");
    }
    *out = n;
    return NRB_OK;
}
}  // namespace nrb

extern "C" nrb_status nrb_nmi_create(int ref_bins, int flo_bins, nrb_nmi **out) {
    return nmi_create_on(ref_bins, flo_bins, nullptr, out);
}

extern "C" void nrb_nmi_destroy(nrb_nmi *nmi) {
    if (!nmi) return;
    dev_free(nmi->hist, nmi->st);
    dev_free(nmi->pro, nmi->st);
    dev_free(nmi->logt, nmi->st);
    dev_free(nmi->last, nmi->st);
    dev_free(nmi->pro2, nmi->st);
    dev_free(nmi->logt2, nmi->st);
    dev_free(nmi->last2, nmi->st);
    delete nmi;
}

extern "C" nrb_status nrb_nmi_read_tables(nrb_nmi *nmi, double *pro_host, double *log_host, double *ent_host,
                                          void *stream) {
    if (!nmi) return fail(NRB_ERR_INVALID, "nrb_nmi_read_tables: null handle");
    cudaStream_t st = as_stream(stream);
    if (pro_host) NRB_CUDA(cudaMemcpyAsync(pro_host, nmi->pro, (size_t)nmi->total * 8, cudaMemcpyDeviceToHost, st));
    if (log_host) NRB_CUDA(cudaMemcpyAsync(log_host, nmi->logt, (size_t)nmi->total * 8, cudaMemcpyDeviceToHost, st));
    nrb_objective o;
    NRB_CUDA(cudaMemcpyAsync(&o, nmi->last, sizeof(o), cudaMemcpyDeviceToHost, st));
    NRB_CUDA(cudaStreamSynchronize(st));
    if (ent_host) memcpy(ent_host, o.entropy, 4 * sizeof(double));
    return NRB_OK;
}

static nrb_status check_fused_args(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g, const float *ref,
                                   const float *flo, const float *cpp) {
    if (!ws || !nmi || !g || !ref || !flo || !cpp) return fail(NRB_ERR_INVALID, "null pointer");
    if (memcmp(&ws->g, g, sizeof(nrb_geometry)) != 0)
        return fail(NRB_ERR_INVALID, "workspace was created for another geometry");
    return NRB_OK;
}

namespace nrb {

nrb_status f3d_objective(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g, const float *ref,
                         const float *flo, int flo_margin, const int32_t *mask, const float *cpp, float padding,
                         double sim_weight, double be_weight, nrb_objective *obj, nrb_objective *obj_host,
                         cudaStream_t st) {
    if (ws->general)
        return fail(NRB_ERR_UNSUPPORTED, "fused evaluation: the grid must be aligned with the reference");
    int n_be = 0;
    const bool overlap = be_weight > 0 && sim_weight > 0;
    if (be_weight > 0) {
        // the bending energy reads only the grid: it runs beside the voxel pass
        if (overlap) NRB_TRY(fork_side(ws, st));
        NRB_TRY(launch_be_value(ws, g, cpp, overlap ? ws->side : st));
        n_be = be_partial_count(g);
    }
    if (sim_weight > 0)
        NRB_TRY(launch_fused_objective(ws, nmi, g, ref, flo, mask, cpp, padding, st, nullptr, nullptr, flo_margin));
    if (overlap) NRB_TRY(join_side(ws, st));
    NRB_TRY(launch_nmi_finalize(nmi, ws->be_partials, n_be, 3 * nvox(g->cpp_dim), sim_weight, be_weight, obj, st));
    if (obj_host) {
        NRB_CUDA(cudaMemcpyAsync(obj_host, obj ? obj : nmi->last, sizeof(nrb_objective), cudaMemcpyDeviceToHost, st));
        NRB_CUDA(cudaStreamSynchronize(st));
    }
    return NRB_OK;
}

nrb_status f3d_gradient(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g, const float *ref,
                        const float *flo, int flo_margin, const int32_t *mask, const float *cpp, float padding,
                        double sim_weight, double be_weight, float *vgrad, float *node_grad, cudaStream_t st) {
    if (ws->general)
        return fail(NRB_ERR_UNSUPPORTED, "fused evaluation: the grid must be aligned with the reference");
    const bool overlap = be_weight > 0 && sim_weight > 0;
    if (overlap) {
        // the bending-energy derivatives read only the grid: they run beside the voxel passes
        NRB_TRY(fork_side(ws, st));
        NRB_TRY(launch_be_derivatives(ws, g, cpp, ws->side));
    }
    if (sim_weight > 0) {
        // the histogram of the current position feeds the log table of the voxel gradient
        NRB_TRY(launch_fused_objective(ws, nmi, g, ref, flo, mask, cpp, padding, st, nullptr, nullptr, flo_margin));
        NRB_TRY(launch_nmi_finalize(nmi, nullptr, 0, 3 * nvox(g->cpp_dim), sim_weight, 0.0, nullptr, st));
        NRB_TRY(launch_fused_gradient(ws, nmi, g, ref, flo, mask, cpp, padding, 1.0, vgrad, st, nullptr, flo_margin));
        NRB_TRY(launch_convolve_to_nodes(ws, g, vgrad, (float)sim_weight, node_grad, st));
    } else {
        NRB_CUDA(cudaMemsetAsync(node_grad, 0, 3 * nvox(g->cpp_dim) * sizeof(float), st));
    }
    if (be_weight > 0) {
        if (overlap) NRB_TRY(join_side(ws, st));
        else NRB_TRY(launch_be_derivatives(ws, g, cpp, st));
        NRB_TRY(launch_be_accumulate(ws, g, (float)be_weight, node_grad, st));
    }
    return NRB_OK;
}

}  // namespace nrb

extern "C" nrb_status nrb_f3d_objective(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g,
                                        const float *ref, const float *flo, const int32_t *mask,
                                        const float *cpp, float padding, double sim_weight,
                                        double be_weight, nrb_objective *obj, nrb_objective *obj_host,
                                        void *stream) {
    NRB_TRY(check_fused_args(ws, nmi, g, ref, flo, cpp));
    return f3d_objective(ws, nmi, g, ref, flo, 0, mask, cpp, padding, sim_weight, be_weight, obj, obj_host,
                         as_stream(stream));
}

extern "C" nrb_status nrb_f3d_gradient(nrb_workspace *ws, nrb_nmi *nmi, const nrb_geometry *g,
                                       const float *ref, const float *flo, const int32_t *mask,
                                       const float *cpp, float padding, double sim_weight,
                                       double be_weight, float *vgrad, float *node_grad, void *stream) {
    NRB_TRY(check_fused_args(ws, nmi, g, ref, flo, cpp));
    if (!vgrad || !node_grad) return fail(NRB_ERR_INVALID, "nrb_f3d_gradient: null buffer");
    return f3d_gradient(ws, nmi, g, ref, flo, 0, mask, cpp, padding, sim_weight, be_weight, vgrad, node_grad,
                        as_stream(stream));
}
