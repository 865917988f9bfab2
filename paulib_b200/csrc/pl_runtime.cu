// pl_runtime.cu -- status reporting and per-device bookkeeping.
//
// The reference reports CUDA failures by throwing std::runtime_error
// (include/gpu/GpuPauliSum.h:25-30) and traps on a bad array size
// (src/gpu/gpu_mul.cu:122-131).  Here every entry point returns a status
// code; the most recent status and a message are kept per host thread so
// the void drop-ins can be checked with pl_get_last_error().

#include <atomic>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "pl_collate.cuh"
#include "pl_common.cuh"

namespace {
thread_local int g_last_status = PL_OK;
thread_local std::string g_last_msg;

std::atomic<unsigned long long> g_launches{0};
std::atomic<bool> g_timing{false};
struct Timed {
    cudaEvent_t start, stop;
    unsigned long long bytes;
    const char* name;
};
std::mutex g_timed_mu;
std::vector<Timed> g_timed;
}  // namespace

namespace pl {

int record_status(int code, const char* what) {
    g_last_status = code;
    if (code == PL_OK) {
        g_last_msg.clear();
    } else {
        g_last_msg = std::string(pl_status_string(code)) + (what ? std::string(": ") + what : "");
    }
    return code;
}

int record_cuda(cudaError_t e) {
    const char* s = cudaGetErrorString(e);
    cudaGetLastError();  // clear a sticky launch error where possible
    g_last_status = e == cudaErrorMemoryAllocation ? PL_ERR_OOM : PL_ERR_CUDA;
    g_last_msg = std::string("CUDA: ") + (s ? s : "unknown error");
    return g_last_status;
}

namespace {
constexpr int kMaxReads = 4;
struct ReadArgs {
    const unsigned int* src[kMaxReads];
    unsigned int dst_off[kMaxReads];
    unsigned int words[kMaxReads];
    int n;
};
// Copies the requested words into the mapped host buffer, then -- after
// every lane's writes are visible system-wide -- writes the call's sequence
// number into the buffer's token word, which the host polls.
__global__ void __launch_bounds__(32) k_readback(ReadArgs a, unsigned int* dst,
                                                 unsigned int* token, unsigned int seq) {
    for (int r = 0; r < a.n; ++r)
        for (unsigned int i = threadIdx.x; i < a.words[r]; i += 32) dst[a.dst_off[r] + i] = a.src[r][i];
    __threadfence_system();
    __syncwarp();
    if (threadIdx.x == 0) *reinterpret_cast<volatile unsigned int*>(token) = seq;
}
struct PinnedBuf {
    void* host = nullptr;
    unsigned int* dev = nullptr;
    size_t bytes = 0;    // data bytes; the token word follows them
    unsigned int seq = 0;
    ~PinnedBuf() {
        if (host) cudaFreeHost(host);
    }
};
thread_local PinnedBuf g_readback;

__global__ void __launch_bounds__(256) k_fill32(unsigned int* p, size_t words, unsigned int v) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if ((reinterpret_cast<uintptr_t>(p) & 15u) == 0) {
        uint4* q = reinterpret_cast<uint4*>(p);
        const size_t n4 = words / 4;
        for (size_t k = i; k < n4; k += stride) q[k] = make_uint4(v, v, v, v);
        for (size_t k = n4 * 4 + i; k < words; k += stride) p[k] = v;
    } else {
        for (size_t k = i; k < words; k += stride) p[k] = v;
    }
}
struct FillArgs {
    unsigned int* p[kMaxFills];
    size_t words[kMaxFills];
    unsigned int v[kMaxFills];
};
// Region blockIdx.y of a multi-region fill.
__global__ void __launch_bounds__(256) k_fill32_multi(FillArgs a) {
    const int r = blockIdx.y;
    unsigned int* p = a.p[r];
    const size_t words = a.words[r];
    const unsigned int v = a.v[r];
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < words; k += stride) p[k] = v;
}
}  // namespace

cudaError_t fill32_multi(const FillReq* reqs, int n, cudaStream_t st) {
    if (n < 1 || n > kMaxFills) return cudaErrorInvalidValue;
    FillArgs a{};
    size_t most = 0;
    for (int r = 0; r < n; ++r) {
        if (reqs[r].bytes % 4 != 0 || (reinterpret_cast<uintptr_t>(reqs[r].p) & 3u) != 0)
            return cudaErrorInvalidValue;
        a.p[r] = static_cast<unsigned int*>(reqs[r].p);
        a.words[r] = reqs[r].bytes / 4;
        a.v[r] = reqs[r].value;
        if (a.words[r] > most) most = a.words[r];
    }
    const int bx = grid_for((i64)(most ? most : 1), 256, sm_count() * 2);
    k_fill32_multi<<<dim3(bx, n), 256, 0, st>>>(a);
    note_launch();
    return cudaGetLastError();
}

cudaError_t readback_sync(const ReadReq* reqs, int n, cudaStream_t st) {
    if (n < 1 || n > kMaxReads) return cudaErrorInvalidValue;
    ReadArgs a{};
    size_t total = 0;
    for (int r = 0; r < n; ++r) {
        if (reqs[r].bytes % 4 != 0 || (reinterpret_cast<uintptr_t>(reqs[r].dev) & 3u) != 0)
            return cudaErrorInvalidValue;
        a.src[r] = static_cast<const unsigned int*>(reqs[r].dev);
        a.dst_off[r] = (unsigned int)(total / 4);
        a.words[r] = (unsigned int)(reqs[r].bytes / 4);
        total += reqs[r].bytes;
    }
    a.n = n;
    PinnedBuf& b = g_readback;
    // one buffer per host thread: every use ends in a stream synchronisation,
    // so no kernel of this thread still writes to it when it is replaced
    if (b.bytes < total) {
        if (b.host) cudaFreeHost(b.host);
        b.host = nullptr;
        b.bytes = 0;
        const size_t want = total < 4096 ? 4096 : (total + 63) & ~size_t(63);
        cudaError_t e =
            cudaHostAlloc(&b.host, want + 64, cudaHostAllocMapped | cudaHostAllocPortable);
        if (e != cudaSuccess) return e;
        void* d = nullptr;
        e = cudaHostGetDevicePointer(&d, b.host, 0);
        if (e != cudaSuccess) return e;
        b.dev = static_cast<unsigned int*>(d);
        b.bytes = want;
        *reinterpret_cast<volatile unsigned int*>(static_cast<unsigned char*>(b.host) + want) = 0;
        b.seq = 0;
    }
    const unsigned int seq = ++b.seq == 0 ? ++b.seq : b.seq;  // never 0 (the initial value)
    unsigned int* dtok = b.dev + b.bytes / 4;
    k_readback<<<1, 32, 0, st>>>(a, b.dev, dtok, seq);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // Wait for the token instead of synchronising the stream: the read-back
    // runs after all earlier work of the stream, so its token means that work
    // is done too.  A poll of host memory needs no driver call; the stream is
    // queried now and then, for errors and in case the token write is not
    // yet visible.  The thread spins (with a pause) rather than yielding: on
    // a busy host a yield can hand the core away for a whole time slice.
    const volatile unsigned int* htok = reinterpret_cast<const volatile unsigned int*>(
        static_cast<const unsigned char*>(b.host) + b.bytes);
    for (unsigned long long i = 1; *htok != seq; ++i) {
        if ((i & 1023u) == 0) {
            e = cudaStreamQuery(st);
            if (e == cudaSuccess) {
                if (*htok == seq) break;
                // completed: the token write must be visible now; one more
                // look, then fall back to the copy as written
                break;
            }
            if (e != cudaErrorNotReady) return e;
        }
#if defined(__x86_64__)
        __builtin_ia32_pause();
#endif
    }
    std::atomic_thread_fence(std::memory_order_acquire);
    const unsigned char* h = static_cast<const unsigned char*>(b.host);
    for (int r = 0; r < n; ++r) std::memcpy(reqs[r].host, h + (size_t)a.dst_off[r] * 4, reqs[r].bytes);
    return cudaSuccess;
}

cudaError_t fill32_async(void* p, unsigned int value, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return cudaSuccess;
    if (bytes % 4 != 0 || (reinterpret_cast<uintptr_t>(p) & 3u) != 0) return cudaErrorInvalidValue;
    const size_t words = bytes / 4;
    const int blocks = grid_for((i64)((words + 3) / 4), 256, sm_count() * 4);
    k_fill32<<<blocks, 256, 0, st>>>(static_cast<unsigned int*>(p), words, value);
    note_launch();
    return cudaGetLastError();
}

static std::mutex g_alloc_mu;
static void keep_pool_cached() {
    static std::mutex mu;
    static std::vector<bool> done;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)done.size() <= dev) done.resize(dev + 1, false);
    if (done[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    done[dev] = true;
}
static std::atomic<long long> g_tuning[16] = {};

// PL_TUNE_FAIL_ALLOC: the k-th allocation from now fails (then the
// injection is spent).
static bool injected_alloc_failure() {
    long long k = g_tuning[PL_TUNE_FAIL_ALLOC].load();
    while (k > 0 && !g_tuning[PL_TUNE_FAIL_ALLOC].compare_exchange_weak(k, k - 1)) {
    }
    return k == 1;
}

cudaError_t dev_alloc(void** p, size_t bytes, cudaStream_t st) {
    keep_pool_cached();
    if (injected_alloc_failure()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    std::lock_guard<std::mutex> lock(g_alloc_mu);
    return cudaMallocAsync(p, bytes, st);
}
void dev_free(void* p, cudaStream_t st) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_alloc_mu);
    cudaFreeAsync(p, st);
}
void capture_lock() { g_alloc_mu.lock(); }
void capture_unlock() { g_alloc_mu.unlock(); }

long long tuning(int key) { return key >= 0 && key < 16 ? g_tuning[key].load() : 0; }

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void note_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
bool timing_enabled() { return g_timing.load(std::memory_order_relaxed); }
void timed_push(cudaEvent_t start, cudaEvent_t stop, unsigned long long bytes, const char* name) {
    std::lock_guard<std::mutex> lock(g_timed_mu);
    g_timed.push_back(Timed{start, stop, bytes, name});
}

cudaEvent_t timed_begin(cudaStream_t st) {
    if (!timing_enabled()) return nullptr;
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    cudaEventRecord(e, st);
    return e;
}

void timed_end(cudaEvent_t start, cudaStream_t st, const char* name, unsigned long long bytes) {
    if (!start) return;
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    cudaEventRecord(e, st);
    timed_push(start, e, bytes, name);
}

int sm_count() {
    static std::mutex mu;
    static std::vector<int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if ((int)cache.size() <= dev) cache.resize(dev + 1, 0);
    if (cache[dev] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
            v = 148;
        cache[dev] = v;
    }
    return cache[dev];
}

}  // namespace pl

extern "C" const char* pl_status_string(int status) {
    switch (status) {
        case PL_OK: return "ok";
        case PL_ERR_INVALID_ARG: return "invalid argument";
        case PL_ERR_OOM: return "out of device memory";
        case PL_ERR_TIMEOUT: return "device wait timed out";
        case PL_ERR_CUDA: return "CUDA error";
        case PL_ERR_CAPACITY: return "output capacity exceeded";
        case PL_ERR_UNSUPPORTED: return "unsupported";
        case PL_ERR_INTERNAL: return "internal consistency check failed";
        case PL_ERR_CANCELLED: return "cancelled";
        default: return "unknown status";
    }
}

extern "C" int pl_get_last_error(void) { return g_last_status; }
extern "C" const char* pl_last_error_message(void) { return g_last_msg.c_str(); }
extern "C" int pl_version(void) { return 1; }

extern "C" int pl_profile_reset(int enable_timing) {
    {
        std::lock_guard<std::mutex> lock(g_timed_mu);
        for (auto& t : g_timed) {
            cudaEventSynchronize(t.stop);
            cudaEventDestroy(t.start);
            cudaEventDestroy(t.stop);
        }
        g_timed.clear();
    }
    g_launches.store(0);
    g_timing.store(enable_timing != 0);
    return pl::record_status(PL_OK, nullptr);
}

extern "C" int pl_profile_read(uint64_t* launches, uint64_t* timed_launches, double* timed_ms,
                               uint64_t* timed_bytes) {
    double ms = 0.0;
    unsigned long long bytes = 0, count = 0;
    {
        std::lock_guard<std::mutex> lock(g_timed_mu);
        for (auto& t : g_timed) {
            if (std::string(t.name) != "k_radix_pass") continue;
            float e = 0.f;
            if (cudaEventSynchronize(t.stop) != cudaSuccess ||
                cudaEventElapsedTime(&e, t.start, t.stop) != cudaSuccess)
                return pl::record_cuda(cudaGetLastError());
            ms += e;
            bytes += t.bytes;
            ++count;
        }
    }
    if (launches) *launches = g_launches.load();
    if (timed_launches) *timed_launches = count;
    if (timed_ms) *timed_ms = ms;
    if (timed_bytes) *timed_bytes = bytes;
    return pl::record_status(PL_OK, nullptr);
}

extern "C" int pl_profile_report(char* buf, size_t cap) {
    // "name count total_ms bytes\n" per kernel name, in first-seen order
    std::vector<std::string> names;
    std::vector<double> ms;
    std::vector<unsigned long long> cnt, bytes;
    {
        std::lock_guard<std::mutex> lock(g_timed_mu);
        for (auto& t : g_timed) {
            float e = 0.f;
            if (cudaEventSynchronize(t.stop) != cudaSuccess ||
                cudaEventElapsedTime(&e, t.start, t.stop) != cudaSuccess)
                return pl::record_cuda(cudaGetLastError());
            size_t k = 0;
            while (k < names.size() && names[k] != t.name) ++k;
            if (k == names.size()) {
                names.push_back(t.name);
                ms.push_back(0.0);
                cnt.push_back(0);
                bytes.push_back(0);
            }
            ms[k] += e;
            cnt[k] += 1;
            bytes[k] += t.bytes;
        }
    }
    std::string out;
    char line[256];
    for (size_t k = 0; k < names.size(); ++k) {
        snprintf(line, sizeof(line), "%s %llu %.6f %llu\n", names[k].c_str(), cnt[k], ms[k],
                 bytes[k]);
        out += line;
    }
    if (!buf || cap == 0) return pl::record_status(PL_ERR_INVALID_ARG, "pl_profile_report");
    snprintf(buf, cap, "%s", out.c_str());
    return pl::record_status(out.size() < cap ? PL_OK : PL_ERR_CAPACITY, nullptr);
}

namespace pl {
cudaError_t set_spin_limit_collate(u32 v);
cudaError_t set_spin_limit_propagate(u32 v);
cudaError_t set_spin_limit_terms(u32 v);
}  // namespace pl

extern "C" int pl_set_tuning(int key, int64_t value) {
    if (key == PL_TUNE_SPIN_LIMIT && value >= 0 && value <= (1ll << 30)) {
        const pl::u32 v = value == 0 ? pl::kSpinLimit : (pl::u32)value;
        PL_CUDA_TRY(pl::set_spin_limit_collate(v));
        PL_CUDA_TRY(pl::set_spin_limit_propagate(v));
        PL_CUDA_TRY(pl::set_spin_limit_terms(v));
        pl::g_tuning[key].store(value);
        return pl::record_status(PL_OK, nullptr);
    }
    if (key == PL_TUNE_FAIL_ALLOC && value >= 0) {
        pl::g_tuning[key].store(value);
        return pl::record_status(PL_OK, nullptr);
    }
    if (key == PL_TUNE_RADIX_BACKOFF && value >= 0 && value <= 1024) {
        pl::g_tuning[key].store(value);
        return pl::record_status(PL_OK, nullptr);
    }
    if (key == PL_TUNE_RADIX_WINDOW &&
        (value == 0 || value == 2 || value == 4 || value == 8 || value == 16)) {
        pl::g_tuning[key].store(value);
        return pl::record_status(PL_OK, nullptr);
    }
    if (key == PL_TUNE_RADIX_ITEMS && (value == 0 || value == 8 || value == 12 || value == 16)) {
        pl::g_tuning[key].store(value);
        return pl::record_status(PL_OK, nullptr);
    }
    if (key == PL_TUNE_RADIX_PREFETCH && value >= -1 && value <= (1 << 20)) {
        pl::g_tuning[key].store(value);
        return pl::record_status(PL_OK, nullptr);
    }
    if ((key == PL_TUNE_INDEX_KEYS || key == PL_TUNE_WINDOW_KEYS || key == PL_TUNE_RADIX_WIDE ||
         key == PL_TUNE_FOLD_GATHER) &&
        (value == 0 || value == 1 || value == -1)) {
        pl::g_tuning[key].store(value);
        return pl::record_status(PL_OK, nullptr);
    }
    return pl::record_status(PL_ERR_INVALID_ARG, "pl_set_tuning");
}

extern "C" int pl_get_tuning(int key, int64_t* value) {
    if (!value || key < 1 || key >= 16) return pl::record_status(PL_ERR_INVALID_ARG, "pl_get_tuning");
    *value = pl::g_tuning[key].load();
    return pl::record_status(PL_OK, nullptr);
}
