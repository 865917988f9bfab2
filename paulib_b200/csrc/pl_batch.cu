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
#include <cmath>
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

// Terms a lane's state is created with (and the floor of every admission
// reserve: a fresh state's five buffers).
constexpr int64_t kFreshTerms = 1 << 16;

size_t term_bytes(int as) { return (size_t)(16 * as + 9); }
size_t fresh_bytes(const pl_job& j) {
    const int64_t n = std::max<int64_t>(j.obs_n, kFreshTerms);
    return 5 * term_bytes(j.array_size) * (size_t)n;
}

// Qubits of the observable's light cone: its support, grown through every
// multi-qubit generator and two-qubit gate it meets, walking the circuit in
// Heisenberg order (last op first).  Single-qubit rotations cannot add a
// qubit: a term only branches when it anticommutes with the generator, i.e.
// already acts on the generator's qubit.
int light_cone(const pl_job& j) {
    const int nq = 64 * j.array_size;
    std::vector<char> in(nq, 0);
    auto add_words = [&](const uint64_t* x, const uint64_t* z, int64_t stride, int64_t t) {
        for (int k = 0; k < j.array_size; ++k) {
            const uint64_t w = x[(size_t)k * stride + t] | z[(size_t)k * stride + t];
            for (int b = 0; b < 64; ++b)
                if ((w >> b) & 1ull) in[64 * k + b] = 1;
        }
    };
    auto touches = [&](const uint64_t* x, const uint64_t* z, int64_t stride, int64_t t) {
        for (int k = 0; k < j.array_size; ++k) {
            const uint64_t w = x[(size_t)k * stride + t] | z[(size_t)k * stride + t];
            for (int b = 0; b < 64; ++b)
                if (((w >> b) & 1ull) && in[64 * k + b]) return true;
        }
        return false;
    };
    for (int64_t t = 0; t < j.obs_n; ++t) add_words(j.obs_x, j.obs_z, j.obs_n, t);
    auto rotation = [&](int64_t r) {
        if (r >= 0 && r < j.n_rot && touches(j.rot_x, j.rot_z, j.n_rot, r))
            add_words(j.rot_x, j.rot_z, j.n_rot, r);
    };
    if (!j.ops) {
        for (int64_t r = j.n_rot; r-- > 0;) rotation(r);
    } else {
        for (int64_t l = j.n_ops; l-- > 0;) {
            const int kind = j.ops[3 * l], a = j.ops[3 * l + 1], b = j.ops[3 * l + 2];
            if (kind == PL_OP_ROTATION) {
                rotation(a);
            } else if (kind == PL_OP_CNOT ||
                       (kind > PL_OP_CLIFFORD && kind - PL_OP_CLIFFORD >= PL_GATE_CNOT)) {
                if (a >= 0 && b >= 0 && a < nq && b < nq && (in[a] || in[b])) in[a] = in[b] = 1;
            }
        }
    }
    int s = 0;
    for (char c : in) s += c;
    return s;
}

// sum_{k <= kmax} C(s, k) 3^k, saturating
long double weight_bound(int s, uint64_t w) {
    const int kmax = (int)std::min<uint64_t>((uint64_t)s, w);
    long double c = 1.0L, sum = 0.0L;
    for (int k = 0; k <= kmax; ++k) {
        sum += c;
        c = c * (long double)(s - k) / (long double)(k + 1) * 3.0L;
    }
    return sum;
}

void estimate(const pl_job& j, uint64_t* terms, uint64_t* bytes) {
    const long double kMax = 1.8e19L;
    long double t = 2.0L * weight_bound(light_cone(j), j.trunc.max_weight);
    const double eps = j.trunc.coefficient_cutoff;
    if (eps > 0.0) {
        long double l1 = 0.0L;
        for (int64_t i = 0; i < j.obs_n; ++i) l1 += std::fabs((long double)j.obs_val[i]);
        const long double fro = 2.0L * l1 * l1 / ((long double)eps * (long double)eps);
        t = std::min(t, std::floor(fro));
    }
    t = std::max(t, (long double)j.obs_n);
    const long double b = 20.0L * (long double)term_bytes(j.array_size) * t + 64.0L * 1048576.0L;
    *terms = t >= kMax ? ~0ull : (uint64_t)t;
    *bytes = b >= kMax ? ~0ull : (uint64_t)b;
}

struct Lane {
    cudaStream_t st = nullptr;
    pl_state* state[kMaxAS + 1] = {};
};

struct Shared {
    const pl_job* jobs = nullptr;
    std::vector<uint64_t> reserve;   // admission reserve per job (bytes)
    std::atomic<uint64_t> rejected{0};
    std::atomic<uint64_t> deferred{0};
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

bool cancelled(const pl_job& job) {
    return job.cancel && *reinterpret_cast<const volatile int32_t*>(job.cancel) != 0;
}

int run_job(Shared& S, Lane& L, const pl_job& job, pl_job_result& r) {
    const int as = job.array_size;
    if (as < 1 || as > kMaxAS) return PL_ERR_INVALID_ARG;
    if (cancelled(job)) return PL_ERR_CANCELLED;
    pl_state*& s = L.state[as];
    int rc = PL_OK;
    if (!s) {
        rc = pl_state_create(&s, as, kFreshTerms, L.st);
        if (rc) return rc;
        state_attach_budget(s, &S.budget);
    }
    rc = pl_state_set_option(s, PL_OPT_GRAPHS, S.opts.use_graphs ? 1 : 0);
    if (rc) return rc;
    rc = pl_state_upload(s, job.obs_x, job.obs_z, job.obs_flags, job.obs_val, job.obs_n);
    if (rc) return rc;
    pl_state_set_cancel_flag(s, job.cancel);
    rc = pl_propagate(s, job.rot_x, job.rot_z, job.rot_flags, job.rot_theta, job.n_rot, job.ops,
                      job.n_ops, &job.trunc);
    pl_state_set_cancel_flag(s, nullptr);
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
        r.lane = lane;
        if (fresh_bytes(S.jobs[j]) > S.budget.limit) {
            // a fresh state for this job alone exceeds the budget: refused
            r.start_s = r.end_s = since(S);
            r.status = PL_ERR_OOM;
            S.rejected.fetch_add(1);
            S.failed.fetch_add(1);
            continue;
        }
        const size_t held = lane_bytes(L);
        const size_t need = S.reserve[(size_t)j] > held ? S.reserve[(size_t)j] - held : 0;
        if (S.budget.admit(need)) S.deferred.fetch_add(1);
        r.start_s = since(S);
        r.status = L.st ? run_job(S, L, S.jobs[j], r) : PL_ERR_CUDA;
        r.end_s = since(S);
        S.budget.leave(need);
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
    // admission reserves: the job's estimate, at most a lane's share of the
    // budget (online growth monitoring covers the rest), at least a fresh
    // state
    S.reserve.resize((size_t)count);
    for (int64_t i = 0; i < count; ++i) {
        uint64_t t = 0, b = 0;
        estimate(jobs[i], &t, &b);
        const size_t share = S.budget.limit / (size_t)opts->lanes;
        S.reserve[(size_t)i] = std::max(fresh_bytes(jobs[i]), std::min<size_t>(b, share));
    }
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
        stats->jobs_rejected = S.rejected.load();
        stats->admission_waits = S.deferred.load();
    }
    if (S.failed.load()) return record_status(PL_ERR_INTERNAL, "batch: a job failed (see results)");
    return record_status(PL_OK, nullptr);
}

}  // namespace
}  // namespace pl

extern "C" int pl_job_estimate(const pl_job* job, uint64_t* terms, uint64_t* bytes) {
    if (!job || !terms || !bytes || job->array_size < 1 || job->array_size > pl::kMaxAS ||
        job->obs_n < 0 || job->n_rot < 0 || job->n_ops < 0 ||
        (job->obs_n > 0 && (!job->obs_x || !job->obs_z || !job->obs_val)) ||
        (job->n_rot > 0 && (!job->rot_x || !job->rot_z)) || (job->n_ops > 0 && !job->ops))
        return pl::record_status(PL_ERR_INVALID_ARG, "pl_job_estimate");
    pl::estimate(*job, terms, bytes);
    return pl::record_status(PL_OK, nullptr);
}

extern "C" int pl_batch_propagate(const pl_job* jobs, int64_t count, const pl_batch_opts* opts,
                                  pl_job_result* results, pl_batch_stats* stats) {
    return pl::run_all(jobs, count, opts, results, stats, false);
}

extern "C" int pl_serve(const pl_job* jobs, int64_t count, const pl_batch_opts* opts,
                        pl_job_result* results, pl_batch_stats* stats) {
    return pl::run_all(jobs, count, opts, results, stats, true);
}
