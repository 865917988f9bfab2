// pl_batch.cu -- many propagations on one device: the batch executor and the
// serving loop (continuous batching).
//
// Each lane is a host thread with its own non-blocking CUDA stream and its
// own device-resident states (one per array size), reused from job to job,
// so buffers, captured graphs and gate tables survive between jobs.  A job
// is propagate_expectation (PauliPropagation.h:65-71) through the C ABI:
// upload, pl_propagate, zero_state_expectation.  The kernels of concurrent
// jobs overlap on the GPU, and the host-side waits of one job (size
// read-backs, the key-mask read of a re-sort) hide behind the work of the
// others.  Every job computes exactly what a lone pl_propagate computes:
// nothing is shared between jobs but the device and the memory budget.
//
// Memory: all lanes' buffers count against one MemBudget.  A lane admits a
// job while the budget is not spent by others; a state that must grow past
// the budget waits until other lanes release memory.  After a job a lane
// gives its buffers back when it holds more than its share (keep_bytes) or
// when another lane is waiting for memory.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

#include "pl_budget.h"
#include "pl_common.cuh"

namespace pl {
void state_attach_budget(pl_state* s, MemBudget* b);
size_t state_held_bytes(pl_state* s);
int state_shrink(pl_state* s);

namespace {

using Clock = std::chrono::steady_clock;

struct Lane {
    cudaStream_t st = nullptr;
    pl_state* state[kMaxAS + 1] = {};
};

struct Shared {
    const pl_job* jobs = nullptr;
    std::vector<int64_t> order;  // job indices in dispatch order
    pl_job_result* results = nullptr;
    pl_batch_opts opts{};
    MemBudget budget;
    Clock::time_point t0;
    bool serving = false;
    std::mutex mu;
    std::condition_variable cv;
    size_t next = 0;             // position in order
    std::atomic<uint64_t> failed{0};
    int device = 0;
};

double since(const Shared& S) {
    return std::chrono::duration<double>(Clock::now() - S.t0).count();
}

// Next job for a lane: -1 when none is left.  Serving waits for arrivals.
int64_t take_job(Shared& S) {
    std::unique_lock<std::mutex> lock(S.mu);
    if (S.next >= S.order.size()) return -1;
    const int64_t j = S.order[S.next];
    if (S.serving) {
        const double wait = S.jobs[j].arrival_s - since(S);
        if (wait > 0) {
            // the earliest job has not arrived: sleep until it does; another
            // lane may take it meanwhile, so re-read afterwards
            S.cv.wait_for(lock, std::chrono::duration<double>(wait));
            if (S.next >= S.order.size()) return -1;
            const int64_t k = S.order[S.next];
            if (S.jobs[k].arrival_s > since(S)) return -2;  // retry
            ++S.next;
            return k;
        }
    }
    ++S.next;
    return j;
}

int run_job(Shared& S, Lane& L, const pl_job& job, pl_job_result& r) {
    const int as = job.array_size;
    if (as < 1 || as > kMaxAS) return PL_ERR_INVALID_ARG;
    pl_state*& s = L.state[as];
    int rc = PL_OK;
    if (!s) {
        rc = pl_state_create(&s, as, 1 << 16, L.st);
        if (rc) return rc;
        state_attach_budget(s, &S.budget);
    }
    rc = pl_state_set_option(s, PL_OPT_GRAPHS, S.opts.use_graphs ? 1 : 0);
    if (rc) return rc;
    rc = pl_state_upload(s, job.obs_x, job.obs_z, job.obs_flags, job.obs_val, job.obs_n);
    if (rc) return rc;
    rc = pl_propagate(s, job.rot_x, job.rot_z, job.rot_flags, job.rot_theta, job.n_rot, job.ops,
                      job.n_ops, &job.trunc);
    if (rc) return rc;
    rc = pl_state_zero_state_expectation(s, &r.expectation);
    if (rc) return rc;
    int64_t n = 0;
    rc = pl_state_size(s, &n);
    r.final_terms = n;
    return rc;
}

size_t lane_bytes(Lane& L) {
    size_t b = 0;
    for (auto* s : L.state)
        if (s) b += state_held_bytes(s);
    return b;
}

void lane_main(Shared& S, int lane) {
    cudaSetDevice(S.device);
    Lane L;
    if (cudaStreamCreateWithFlags(&L.st, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        L.st = nullptr;
    }
    const size_t keep = S.opts.keep_bytes ? (size_t)S.opts.keep_bytes
                                          : (size_t)(S.budget.limit / std::max(1, S.opts.lanes));
    for (;;) {
        const int64_t j = take_job(S);
        if (j == -1) break;
        if (j == -2) continue;
        pl_job_result& r = S.results[j];
        S.budget.admit();
        r.lane = lane;
        r.start_s = since(S);
        r.status = L.st ? run_job(S, L, S.jobs[j], r) : PL_ERR_CUDA;
        r.end_s = since(S);
        S.budget.leave();
        if (r.status != PL_OK) S.failed.fetch_add(1);
        // give memory back when over the lane's share or when others wait
        bool others_wait;
        {
            std::lock_guard<std::mutex> lock(S.budget.mu);
            others_wait = S.budget.waiting > 0;
        }
        if (lane_bytes(L) > keep || others_wait)
            for (auto* s : L.state)
                if (s && state_held_bytes(s) > ((size_t)64 << 20)) state_shrink(s);
    }
    for (auto*& s : L.state) {
        if (s) pl_state_destroy(s);
        s = nullptr;
    }
    if (L.st) cudaStreamDestroy(L.st);
}

double job_cost(const pl_job& j) { return (double)j.n_rot * j.array_size; }

int run_all(const pl_job* jobs, int64_t count, const pl_batch_opts* opts, pl_job_result* results,
            pl_batch_stats* stats, bool serving) {
    if (!jobs || count < 0 || !opts || !results || opts->lanes < 1 || opts->lanes > 256)
        return record_status(PL_ERR_INVALID_ARG, "batch: jobs, results or lanes");
    for (int64_t i = 0; i < count; ++i) {
        const pl_job& j = jobs[i];
        if (j.array_size < 1 || j.array_size > kMaxAS || j.obs_n < 0 || j.n_rot < 0 ||
            j.n_ops < 0 || (serving && !(j.arrival_s >= 0.0)))
            return record_status(PL_ERR_INVALID_ARG, "batch: job fields");
        results[i] = pl_job_result{0.0, 0, PL_OK, -1, 0.0, 0.0};
    }
    if (opts->sync_stream) PL_CUDA_TRY(cudaStreamSynchronize(opts->sync_stream));
    Shared S;
    S.jobs = jobs;
    S.results = results;
    S.opts = *opts;
    S.serving = serving;
    PL_CUDA_TRY(cudaGetDevice(&S.device));
    size_t free_b = 0, total_b = 0;
    PL_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    S.budget.limit = opts->hbm_budget ? (size_t)opts->hbm_budget : (size_t)(0.85 * free_b);
    S.order.resize((size_t)count);
    for (int64_t i = 0; i < count; ++i) S.order[(size_t)i] = i;
    if (serving) {
        std::stable_sort(S.order.begin(), S.order.end(), [&](int64_t a, int64_t b) {
            return jobs[a].arrival_s < jobs[b].arrival_s;
        });
    } else if (opts->order == PL_ORDER_LONGEST_FIRST) {
        std::stable_sort(S.order.begin(), S.order.end(), [&](int64_t a, int64_t b) {
            return job_cost(jobs[a]) > job_cost(jobs[b]);
        });
    }
    S.t0 = Clock::now();
    std::vector<std::thread> threads;
    threads.reserve((size_t)opts->lanes);
    for (int l = 0; l < opts->lanes; ++l) threads.emplace_back(lane_main, std::ref(S), l);
    for (auto& t : threads) t.join();
    const double wall = since(S);
    // hand the lanes' cached blocks back to the device
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, S.device) == cudaSuccess) {
        cudaDeviceSynchronize();
        cudaMemPoolTrimTo(pool, 0);
    }
    cudaGetLastError();
    if (stats) {
        stats->wall_s = wall;
        stats->peak_bytes = S.budget.peak;
        stats->budget_waits = S.budget.waits;
        stats->jobs_failed = S.failed.load();
    }
    if (S.failed.load()) return record_status(PL_ERR_INTERNAL, "batch: a job failed (see results)");
    return record_status(PL_OK, nullptr);
}

}  // namespace
}  // namespace pl

extern "C" int pl_batch_propagate(const pl_job* jobs, int64_t count, const pl_batch_opts* opts,
                                  pl_job_result* results, pl_batch_stats* stats) {
    return pl::run_all(jobs, count, opts, results, stats, false);
}

extern "C" int pl_serve(const pl_job* jobs, int64_t count, const pl_batch_opts* opts,
                        pl_job_result* results, pl_batch_stats* stats) {
    return pl::run_all(jobs, count, opts, results, stats, true);
}
