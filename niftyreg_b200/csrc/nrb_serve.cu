// Batched and served F3D registrations on one device.
//
// A server owns `slots` worker threads, each with its own CUDA stream; a worker runs one group of
// requests at a time through the batched registration (one graph per pyramid level in which every
// stage is one launch over all the group's pairs). Requests queue in arrival order. When a worker
// is free and the queue's head fits in what the HBM budget has left, the worker takes the head and
// the queued requests that can share its group (the same parameters, a volume within a factor of
// two of the head's, in arrival order, up to `max_group` requests and the budget). Requests that
// arrive while groups run wait for the next free worker and run beside the groups already on the
// device. Each pair's arithmetic in a group is that of its plain registration, so every result
// equals nrb_f3d_register_host's for the same request alone, whatever it was grouped with.
//
// The batch entry point forms groups the same way from the pairs it is given and runs them on
// two such workers when they fit in half the budget each.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <system_error>
#include <thread>
#include <vector>

#include "nrb_state.cuh"

namespace nrb {
nrb_status register_on_stream(const float *ref, const float *flo, const int32_t dim[3], const float pixdim[3],
                              const nrb_f3d_params *p, float *cpp_out, int64_t cap, nrb_f3d_result *res,
                              cudaStream_t st);
int64_t registration_footprint(const int32_t dim[3], const float pixdim[3], const nrb_f3d_params *p);
}  // namespace nrb

using namespace nrb;
using Clock = std::chrono::steady_clock;

namespace {

struct Job {
    int64_t ticket = 0;
    nrb_pair pair{};
    nrb_f3d_params params{};
    int64_t footprint = 0;
    Clock::time_point submitted, started, finished;
    bool done = false;
    bool claimed = false;  // a nrb_server_wait call owns this ticket
    nrb_status status = NRB_OK;
    std::string error;
    nrb_f3d_result result{};
};

// The library's memory pool on the device (not the application's default pool). While servers
// exist on a device, its release threshold and internal-dependency reuse are set for them; the
// values found when the first server was created are put back when the last one is destroyed.
struct PoolSettings {
    int servers = 0;
    uint64_t threshold = 0;
    int reuse_internal = 1;
};
std::mutex g_pool_mu;
std::map<int, PoolSettings> g_pool_saved;

void pool_acquire(int dev, int64_t budget) {
    cudaMemPool_t pool = lib_pool_of(dev);
    if (!pool) return;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    PoolSettings& ps = g_pool_saved[dev];
    if (ps.servers++ == 0) {
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &ps.threshold);
        cudaMemPoolGetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &ps.reuse_internal);
    }
    // keep freed registration buffers in the pool up to the budget, so the next admitted request
    // reuses them instead of mapping new memory
    uint64_t thr = 0;
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    thr = std::max(thr, (uint64_t)budget);
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    // no reuse across streams through inserted dependencies: a registration must never wait for
    // another one's stream because the pool handed it memory that stream freed
    int no = 0;
    cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no);
    cudaGetLastError();
}

void pool_release(int dev) {
    cudaMemPool_t pool = lib_pool_of(dev);
    if (!pool) return;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    auto it = g_pool_saved.find(dev);
    if (it == g_pool_saved.end() || --it->second.servers > 0) return;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &it->second.threshold);
    cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &it->second.reuse_internal);
    g_pool_saved.erase(it);
    cudaGetLastError();
}

}  // namespace

// parameters two requests must share to run in one group
static bool same_params(const nrb_f3d_params& a, const nrb_f3d_params& b) {
    auto feq = [](float x, float y) { return x == y || (x != x && y != y); };
    for (int i = 0; i < 3; ++i)
        if (!feq(a.spacing[i], b.spacing[i])) return false;
    return a.levels == b.levels && a.max_iterations == b.max_iterations && feq(a.bending_energy, b.bending_energy) &&
           a.ref_bins == b.ref_bins && a.flo_bins == b.flo_bins && feq(a.padding, b.padding) &&
           a.floating_margin == b.floating_margin && a.batch_gradient_percent == b.batch_gradient_percent &&
           a.floating_texture == b.floating_texture && a.verbose == b.verbose && a.autotune == b.autotune &&
           a.batch_group_mb == b.batch_group_mb;
}

static int64_t voxels_of(const nrb_pair& p) { return (int64_t)p.dim[0] * p.dim[1] * p.dim[2]; }
// finest-level reference + floating bytes of a pair (one geometry for both)
static int64_t image_bytes(const nrb_pair& p) { return 2 * 4 * voxels_of(p); }

struct nrb_server {
    int device = 0;
    int64_t budget = 0;
    int max_group = 16;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Job *> queue;
    std::map<int64_t, Job *> jobs;
    std::vector<std::thread> workers;
    int64_t next_ticket = 1, used = 0, peak_used = 0;
    int active = 0, peak_active = 0, peak_group = 0;
    bool stop = false;

    // the head of the queue fits in the budget (always admitted when nothing runs, so a request
    // the size of the whole budget still runs)
    bool head_fits() const { return active == 0 || used + queue.front()->footprint <= budget; }

    // the head and the queued requests that can share its group, removed from the queue
    std::vector<Job *> take_group() {
        std::vector<Job *> g;
        Job *head = queue.front();
        queue.pop_front();
        g.push_back(head);
        int64_t bytes = head->footprint, images = image_bytes(head->pair);
        const int64_t hv = voxels_of(head->pair);
        const int64_t group_bytes = (int64_t)std::max(0, head->params.batch_group_mb) << 20;
        for (auto it = queue.begin(); it != queue.end() && (int)g.size() < max_group;) {
            Job *j = *it;
            const int64_t v = voxels_of(j->pair);
            if (same_params(j->params, head->params) && v <= 2 * hv && hv <= 2 * v &&
                used + bytes + j->footprint <= budget &&
                (group_bytes == 0 || images + image_bytes(j->pair) <= group_bytes)) {
                g.push_back(j);
                bytes += j->footprint;
                images += image_bytes(j->pair);
                it = queue.erase(it);
            } else {
                ++it;
            }
        }
        return g;
    }

    void worker() {
        cudaSetDevice(device);
        cudaStream_t st = nullptr;
        const bool have_stream = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess;
        for (;;) {
            std::vector<Job *> group;
            {
                std::unique_lock<std::mutex> lock(mu);
                // FIFO admission: the head waits for memory rather than being overtaken
                cv.wait(lock, [&] { return (stop && queue.empty()) || (!queue.empty() && head_fits()); });
                if (queue.empty()) break;  // stopping and drained
                group = take_group();
                for (Job *j : group) used += j->footprint;
                active += (int)group.size();
                peak_used = std::max(peak_used, used);
                peak_active = std::max(peak_active, active);
                peak_group = std::max(peak_group, (int)group.size());
            }
            const auto started = Clock::now();
            std::vector<nrb_pair> pairs;
            std::vector<nrb_f3d_result> results(group.size());
            for (Job *j : group) {
                j->started = started;
                pairs.push_back(j->pair);
            }
            nrb_status s = have_stream ? NRB_OK : fail(NRB_ERR_CUDA, "server: stream creation failed");
            if (s == NRB_OK)
                s = register_batch_fused(pairs.data(), (int)pairs.size(), &group[0]->params, results.data(), st,
                                         group[0]->params.batch_gradient_percent);
            const std::string err = s == NRB_OK ? std::string() : std::string(nrb_last_error());
            {
                std::lock_guard<std::mutex> lock(mu);
                const auto finished = Clock::now();
                for (size_t i = 0; i < group.size(); ++i) {
                    Job *j = group[i];
                    j->finished = finished;
                    j->status = s;
                    j->error = err;
                    j->result = results[i];
                    j->done = true;
                    used -= j->footprint;
                }
                active -= (int)group.size();
            }
            cv.notify_all();
        }
        if (st) cudaStreamDestroy(st);
    }
};

extern "C" nrb_status nrb_f3d_footprint(const int32_t dim[3], const float pixdim[3], const nrb_f3d_params *p,
                                        int64_t *bytes) {
    if (!dim || !pixdim || !p || !bytes) return fail(NRB_ERR_INVALID, "nrb_f3d_footprint: null pointer");
    *bytes = registration_footprint(dim, pixdim, p);
    return NRB_OK;
}

extern "C" nrb_status nrb_server_create(int slots, int64_t hbm_budget_bytes, nrb_server **out) {
    return nrb_server_create_grouped(slots, 16, hbm_budget_bytes, out);
}

extern "C" nrb_status nrb_server_create_grouped(int slots, int max_group, int64_t hbm_budget_bytes, nrb_server **out) {
    if (!out || slots < 1 || slots > 256) return fail(NRB_ERR_INVALID, "nrb_server_create: slots must be in [1, 256]");
    if (max_group < 1 || max_group > BATCH_MAX_PAIRS)
        return fail(NRB_ERR_INVALID, "nrb_server_create: max_group must be in [1, " + std::to_string(BATCH_MAX_PAIRS) + "]");
    int dev = 0;
    NRB_CUDA(cudaGetDevice(&dev));
    size_t free_b = 0, total_b = 0;
    NRB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    nrb_server *s = new nrb_server();
    s->device = dev;
    s->max_group = max_group;
    s->budget = hbm_budget_bytes > 0 ? hbm_budget_bytes : (int64_t)(0.8 * (double)free_b);
    pool_acquire(dev, s->budget);
    try {
        for (int i = 0; i < slots; ++i) s->workers.emplace_back([s] { s->worker(); });
    } catch (const std::system_error&) {
        nrb_server_destroy(s);  // stops and joins the workers already started
        return fail(NRB_ERR_INVALID, "nrb_server_create: could not start " + std::to_string(slots) + " worker threads");
    }
    *out = s;
    return NRB_OK;
}

extern "C" nrb_status nrb_server_submit(nrb_server *s, const nrb_pair *req, const nrb_f3d_params *p,
                                        int64_t *ticket) {
    if (!s || !req || !p || !ticket || !req->ref_host || !req->flo_host)
        return fail(NRB_ERR_INVALID, "nrb_server_submit: null pointer");
    for (int i = 0; i < 3; ++i)
        if (req->dim[i] < 2 || !(req->pixdim[i] > 0))
            return fail(NRB_ERR_INVALID, "nrb_server_submit: 3D volumes with positive voxel size expected");
    Job *job = new Job();
    job->pair = *req;
    job->params = *p;
    job->footprint = registration_footprint(req->dim, req->pixdim, p);
    if (p->batch_gradient_percent < 1 || p->batch_gradient_percent > 100) {
        delete job;
        return fail(NRB_ERR_INVALID, "nrb_server_submit: batch_gradient_percent in [1, 100]");
    }
    if (job->footprint > s->budget) {
        delete job;
        return fail(NRB_ERR_OOM, "nrb_server_submit: request larger than the server's HBM budget");
    }
    job->submitted = Clock::now();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        job->ticket = s->next_ticket++;
        s->jobs[job->ticket] = job;
        s->queue.push_back(job);
    }
    s->cv.notify_all();
    *ticket = job->ticket;
    return NRB_OK;
}

extern "C" nrb_status nrb_server_wait(nrb_server *s, int64_t ticket, nrb_f3d_result *res, double *queue_seconds,
                                      double *latency_seconds) {
    if (!s) return fail(NRB_ERR_INVALID, "nrb_server_wait: null server");
    Job *job = nullptr;
    {
        std::unique_lock<std::mutex> lock(s->mu);
        auto it = s->jobs.find(ticket);
        if (it == s->jobs.end()) return fail(NRB_ERR_INVALID, "nrb_server_wait: unknown ticket");
        job = it->second;
        // a ticket is waited on once: a second waiter (another thread) is refused instead of
        // reading the job after the first one has released it
        if (job->claimed) return fail(NRB_ERR_INVALID, "nrb_server_wait: ticket already being waited on");
        job->claimed = true;
        s->cv.wait(lock, [&] { return job->done; });
        s->jobs.erase(ticket);
    }
    const nrb_status st = job->status;
    const std::string err = job->error;
    if (res) *res = job->result;
    if (queue_seconds) *queue_seconds = std::chrono::duration<double>(job->started - job->submitted).count();
    if (latency_seconds) *latency_seconds = std::chrono::duration<double>(job->finished - job->submitted).count();
    delete job;
    if (st != NRB_OK) return fail(st, err.c_str());
    return NRB_OK;
}

extern "C" nrb_status nrb_server_stats(nrb_server *s, int64_t *peak_bytes, int32_t *peak_active) {
    if (!s) return fail(NRB_ERR_INVALID, "nrb_server_stats: null server");
    std::lock_guard<std::mutex> lock(s->mu);
    if (peak_bytes) *peak_bytes = s->peak_used;
    if (peak_active) *peak_active = s->peak_active;
    return NRB_OK;
}

extern "C" nrb_status nrb_server_peak_group(nrb_server *s, int32_t *peak_group) {
    if (!s || !peak_group) return fail(NRB_ERR_INVALID, "nrb_server_peak_group: null pointer");
    std::lock_guard<std::mutex> lock(s->mu);
    *peak_group = s->peak_group;
    return NRB_OK;
}

extern "C" void nrb_server_destroy(nrb_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    for (auto& t : s->workers) t.join();
    for (auto& kv : s->jobs) delete kv.second;
    pool_release(s->device);
    delete s;
}

extern "C" nrb_status nrb_f3d_register_batch(const nrb_pair *pairs, int n, const nrb_f3d_params *p, int concurrency,
                                             int64_t hbm_budget_bytes, nrb_f3d_result *results) {
    if (!pairs || n < 0 || !p) return fail(NRB_ERR_INVALID, "nrb_f3d_register_batch: bad argument");
    if (n == 0) return NRB_OK;
    for (int i = 0; i < n; ++i) {
        if (!pairs[i].ref_host || !pairs[i].flo_host) return fail(NRB_ERR_INVALID, "nrb_f3d_register_batch: null image");
        for (int k = 0; k < 3; ++k)
            if (pairs[i].dim[k] < 2 || !(pairs[i].pixdim[k] > 0))
                return fail(NRB_ERR_INVALID, "nrb_f3d_register_batch: 3D volumes with positive voxel size expected");
    }
    const int pct = p->batch_gradient_percent;
    if (pct < 1 || pct > 100) return fail(NRB_ERR_INVALID, "nrb_f3d_register_batch: batch_gradient_percent in [1, 100]");
    const int group_max = std::max(1, std::min(concurrency > 0 ? concurrency : BATCH_MAX_PAIRS, BATCH_MAX_PAIRS));
    int64_t budget = hbm_budget_bytes;
    if (budget <= 0) {
        size_t free_b = 0, total_b = 0;
        NRB_CUDA(cudaMemGetInfo(&free_b, &total_b));
        budget = (int64_t)(0.8 * (double)free_b);
    }
    // pairs in order of size (stable), so that a group holds pairs of similar size
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return voxels_of(pairs[a]) < voxels_of(pairs[b]); });
    const int64_t group_bytes = (int64_t)std::max(0, p->batch_group_mb) << 20;
    // the groups: pairs while they fit in the group budget (a pair larger than it alone is
    // refused) and their finest-level images in the group cap (the first pair always joins)
    auto plan = [&](int64_t gbudget, std::vector<std::pair<int, int>>& groups) {
        groups.clear();
        for (int i0 = 0; i0 < n;) {
            int64_t used = 0, images = 0;
            int i1 = i0;
            while (i1 < n && i1 - i0 < group_max) {
                const nrb_pair& q = pairs[order[i1]];
                const int64_t f = registration_footprint(q.dim, q.pixdim, p);
                const int64_t img = image_bytes(q);
                if (used + f > gbudget) break;
                if (i1 > i0 && group_bytes > 0 && images + img > group_bytes) break;
                used += f;
                images += img;
                ++i1;
            }
            if (i1 == i0) return false;
            groups.emplace_back(i0, i1);
            i0 = i1;
        }
        return true;
    };
    // two workers, each with half the budget, when that still makes groups and there are two or
    // more: one group's uploads, pyramids and level set-up (host work) overlap the other's
    // graphs on the device. Otherwise one worker with the whole budget.
    std::vector<std::pair<int, int>> groups;
    int workers = 2;
    if (!plan(budget / 2, groups) || groups.size() < 2) {
        workers = 1;
        if (!plan(budget, groups)) return fail(NRB_ERR_OOM, "nrb_f3d_register_batch: a pair is larger than the HBM budget");
    }
    int device = 0;
    NRB_CUDA(cudaGetDevice(&device));
    std::mutex mu;
    size_t next = 0;
    nrb_status first_error = NRB_OK;
    std::string first_message;
    auto work = [&]() {
        cudaStream_t st = nullptr;
        nrb_status s = NRB_OK;
        // the caller's device (a new host thread starts on device 0)
        if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            s = fail(NRB_ERR_CUDA, "nrb_f3d_register_batch: stream creation failed");
        }
        std::vector<nrb_pair> gp;
        std::vector<nrb_f3d_result> gr;
        while (s == NRB_OK) {
            size_t g;
            {
                std::lock_guard<std::mutex> lock(mu);
                if (first_error != NRB_OK || next >= groups.size()) break;
                g = next++;
            }
            const int i0 = groups[g].first, i1 = groups[g].second;
            gp.clear();
            for (int i = i0; i < i1; ++i) gp.push_back(pairs[order[i]]);
            gr.assign(i1 - i0, nrb_f3d_result{});
            s = register_batch_fused(gp.data(), i1 - i0, p, gr.data(), st, pct);
            if (s == NRB_OK && results)
                for (int i = i0; i < i1; ++i) results[order[i]] = gr[i - i0];
        }
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        if (s != NRB_OK) {
            std::lock_guard<std::mutex> lock(mu);
            if (first_error == NRB_OK) {
                first_error = s;
                first_message = nrb_last_error();
            }
        }
    };
    std::thread other;
    if (workers == 2) {
        try {
            other = std::thread(work);
        } catch (const std::system_error&) {
            // no second thread: this one takes every group (the halves of the budget still fit)
        }
    }
    work();
    if (other.joinable()) other.join();
    if (first_error != NRB_OK) return fail(first_error, first_message);
    return NRB_OK;
}
