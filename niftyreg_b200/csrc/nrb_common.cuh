// Internal helpers shared by the niftyreg_b200 CUDA sources (not part of the public ABI).
#pragma once

#include <utility>

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>

#include "niftyreg_b200.h"

namespace nrb {

// ------------------------------------------------------------------------------------------
// error state and launch accounting
// ------------------------------------------------------------------------------------------
void set_error(const std::string& msg);
nrb_status fail(nrb_status code, const std::string& msg);
nrb_status check_cuda(cudaError_t e, const char *what);
extern std::atomic<long long> g_launch_count;

// Call after every kernel launch: counts it and turns a launch error into a status.
#define NRB_LAUNCHED(what)                                                   \
    do {                                                                     \
        ::nrb::g_launch_count.fetch_add(1, std::memory_order_relaxed);       \
        cudaError_t e_ = cudaGetLastError();                                 \
        if (e_ != cudaSuccess) return ::nrb::check_cuda(e_, what);           \
    } while (0)

#define NRB_TRY(expr)                                                        \
    do {                                                                     \
        nrb_status s_ = (expr);                                              \
        if (s_ != NRB_OK) return s_;                                         \
    } while (0)

#define NRB_CUDA(expr)                                                       \
    do {                                                                     \
        cudaError_t e_ = (expr);                                             \
        if (e_ != cudaSuccess) return ::nrb::check_cuda(e_, #expr);          \
    } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Programmatic dependent launch: a kernel launched with programmatic stream serialization may
// start while its predecessor's last blocks are still running; it must wait here before it reads
// anything the predecessor writes. Without that launch attribute the wait returns at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// Lets the launch that depends on this one (programmatic stream serialization) be scheduled now:
// its blocks may start and do whatever does not need this launch's results, then pdl_wait().
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" :::); }

// cudaLaunchKernelEx with programmatic stream serialization when `pdl` is set.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t st, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// The library's own stream-ordered memory pool on the current device (created on first use;
// null if it cannot be created, and the device's default pool serves instead). Its release
// threshold starts at kLibPoolFloor, so memory freed between calls stays mapped for the next
// ones, and lib_pool_keep raises it; the application's default pool is never changed.
constexpr uint64_t kLibPoolFloor = uint64_t(256) << 20;
cudaMemPool_t lib_pool();
cudaMemPool_t lib_pool_of(int device);
void lib_pool_keep(uint64_t bytes);

// Device allocation tied to an owner's stream: stream-ordered from the library's pool (no
// device-wide synchronisation, so registrations on other streams keep running) when `st` is set,
// plain otherwise.
template <typename T>
inline cudaError_t dev_alloc(T **p, size_t bytes, cudaStream_t st) {
    if (!st) return cudaMalloc(reinterpret_cast<void **>(p), bytes);
    cudaMemPool_t pool = lib_pool();
    return pool ? cudaMallocFromPoolAsync(reinterpret_cast<void **>(p), bytes, pool, st)
                : cudaMallocAsync(reinterpret_cast<void **>(p), bytes, st);
}
// A call's temporary, stream-ordered from the library's pool on any stream (the legacy default
// stream included); released with dev_free(p, st) or cudaFreeAsync on the same stream.
template <typename T>
inline cudaError_t tmp_alloc(T **p, size_t bytes, cudaStream_t st) {
    cudaMemPool_t pool = lib_pool();
    return pool ? cudaMallocFromPoolAsync(reinterpret_cast<void **>(p), bytes, pool, st)
                : cudaMallocAsync(reinterpret_cast<void **>(p), bytes, st);
}
inline void dev_free(void *p, cudaStream_t st) {
    if (!p) return;
    if (st) cudaFreeAsync(p, st);
    else cudaFree(p);
}

// Optional per-kernel CUDA-event timing (nrb_timing_enable). A KernelTimer brackets one launch
// with events on its stream and records the algorithmic bytes that launch must move.
enum TimedKernel {
    TK_OBJECTIVE = 0, TK_GRADIENT, TK_FINALIZE, TK_CONV, TK_BE_VALUE, TK_BE_GRADIENT,
    // F3D2 stages (a stage brackets all launches it makes on its stream) and kernels
    TK_F2_VELOCITY, TK_F2_COMPOSE, TK_F2_GRADIENT_EXP, TK_F2_WARP, TK_F2_NMI, TK_F2_VOXEL_GRADIENT, TK_F2_NODES,
    TK_F2_BE, TK_F2_UPDATE, TK_COUNT
};
class KernelTimer {
public:
    KernelTimer(TimedKernel k, double bytes, cudaStream_t st);
    ~KernelTimer();
private:
    TimedKernel k_;
    double bytes_;
    cudaStream_t st_;
    cudaEvent_t a_ = nullptr;
};

// True while nrb_timing_enable(1) is in force (launch sequences that are captured into CUDA
// graphs then run eagerly instead, so each launch keeps its events).
bool timing_enabled();

// Number of SMs of the current device (cached per device).
int sm_count();

// ------------------------------------------------------------------------------------------
// device-side geometry
// ------------------------------------------------------------------------------------------
struct Mat34 {  // the first three rows of a NIfTI mat44
    float m[12];
};

inline Mat34 to_mat34(const float *m16) {
    Mat34 r;
    for (int i = 0; i < 12; ++i) r.m[i] = m16[i];
    return r;
}

__host__ __device__ inline void mat34_apply(const Mat34& M, float x, float y, float z, float& ox,
                                            float& oy, float& oz) {
    ox = M.m[0] * x + M.m[1] * y + M.m[2] * z + M.m[3];
    oy = M.m[4] * x + M.m[5] * y + M.m[6] * z + M.m[7];
    oz = M.m[8] * x + M.m[9] * y + M.m[10] * z + M.m[11];
}

// Cubic B-spline basis at fractional offset t in [0, 1): weights of nodes pre..pre+3
// (reg-lib/cpu/_reg_splineBasis.cpp:17-26 evaluates the same polynomials).
__host__ __device__ inline void bspline_basis(float t, float b[4]) {
    const float ff = t * t, fff = ff * t, mf = 1.f - t;
    b[0] = mf * mf * mf * (1.f / 6.f);
    b[1] = (3.f * fff - 6.f * ff + 4.f) * (1.f / 6.f);
    b[2] = (-3.f * fff + 3.f * ff + 3.f * t + 1.f) * (1.f / 6.f);
    b[3] = fff * (1.f / 6.f);
}

// Parzen window: cubic B-spline and its derivative (reg-lib/cpu/_reg_nmi.h:116-145). The
// centre constant is float(2/3) exactly as the reference writes it (2.f/3.f).
__host__ __device__ inline double parzen(double x) {
    x = x < 0 ? -x : x;
    if (x < 2.0) {
        if (x < 1.0) return (double)(2.0f / 3.0f) + (0.5 * x - 1.0) * x * x;
        x -= 2.0;
        return -x * x * x / 6.0;
    }
    return 0.0;
}
__host__ __device__ inline double parzen_deriv(double ox) {
    double x = ox < 0 ? -ox : ox;
    if (x < 2.0) {
        if (x < 1.0) return (1.5 * x - 2.0) * ox;
        x -= 2.0;
        const double v = -0.5 * x * x;
        return ox < 0 ? -v : v;
    }
    return 0.0;
}
__device__ inline float parzenf(float x) {
    x = fabsf(x);
    if (x < 2.f) {
        if (x < 1.f) return (2.0f / 3.0f) + (0.5f * x - 1.f) * x * x;
        x -= 2.f;
        return -x * x * x * (1.f / 6.f);
    }
    return 0.f;
}
__device__ inline float parzen_derivf(float ox) {
    float x = fabsf(ox);
    if (x < 2.f) {
        if (x < 1.f) return (1.5f * x - 2.f) * ox;
        x -= 2.f;
        const float v = -0.5f * x * x;
        return ox < 0 ? -v : v;
    }
    return 0.f;
}

inline int64_t nvox(const int32_t d[3]) { return (int64_t)d[0] * d[1] * d[2]; }

// ------------------------------------------------------------------------------------------
// cross-file launchers
// ------------------------------------------------------------------------------------------
// Workspace of scratch buffers sized for one geometry (owned by nrb_workspace).
struct Workspace;
nrb_status be_value_partials(Workspace *ws, const nrb_geometry *g, const float *cpp,
                             cudaStream_t st);
nrb_status be_value_finish(Workspace *ws, nrb_objective *obj, double *be_host, cudaStream_t st);

}  // namespace nrb
