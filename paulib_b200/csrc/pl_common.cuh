// pl_common.cuh -- shared device helpers for the sm_100a Pauli-sum kernels.
//
// Term layout in HBM (same planes as the reference GPU seam,
// include/gpu/GpuPauliSum.h:8-12): x[k*stride + i], z[k*stride + i] for word
// k of term i, flags[i] (bit0 = imaginary, bit1 = sign; exponent of i^k),
// val[i] FP64.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "paulib_b200.h"

namespace pl {

using u64 = unsigned long long;
using u32 = unsigned int;
using u16 = unsigned short;
using u8 = unsigned char;
using i64 = long long;

constexpr int kMaxAS = 16;
// Bound on every spin-wait (decoupled look-back): after this many polls a
// kernel records PL_ERR_TIMEOUT, publishes what it has and moves on.  The
// bound in force is g_spin_limit (PL_TUNE_SPIN_LIMIT; kSpinLimit by
// default): every translation unit that waits holds its own copy, which
// pl_set_tuning writes for the current device through the unit's
// PL_SPIN_LIMIT_SETTER function.
constexpr u32 kSpinLimit = 1u << 20;
static __device__ u32 g_spin_limit = kSpinLimit;
#define PL_SPIN_LIMIT_SETTER(name) \
    cudaError_t name(u32 v) { return cudaMemcpyToSymbol(g_spin_limit, &v, sizeof(v)); }

// ---------------------------------------------------------------------------
// Device status word: the first non-zero code wins.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void raise_status(int* status, int code) {
    if (status) atomicCAS(status, 0, code);
}

__device__ __forceinline__ u32 ld_volatile(const u32* p) {
    return *reinterpret_cast<const volatile u32*>(p);
}
__device__ __forceinline__ u64 ld_volatile64(const u64* p) {
    return *reinterpret_cast<const volatile u64*>(p);
}
__device__ __forceinline__ void st_volatile(u32* p, u32 v) {
    *reinterpret_cast<volatile u32*>(p) = v;
}
__device__ __forceinline__ void st_volatile64(u64* p, u64 v) {
    *reinterpret_cast<volatile u64*>(p) = v;
}

__device__ __forceinline__ u32 lanemask_lt() {
    u32 m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---------------------------------------------------------------------------
// Pauli algebra on packed words.
// Symplectic product, PauliStringCore.h:150-174: per word
//   xbz = ax & bz; anti = (bx & az) ^ xbz;
//   c2 ^= (c1 ^ ax ^ az ^ bx ^ bz ^ xbz) & anti; c1 ^= anti;
// exponent = (fa + fb + popc(c1) + 2*parity(c2)) mod 4.
// ---------------------------------------------------------------------------
struct PhaseAcc {
    u64 c1 = 0, c2 = 0;
    __device__ __forceinline__ void step(u64 ax, u64 az, u64 bx, u64 bz) {
        const u64 xbz = ax & bz;
        const u64 anti = (bx & az) ^ xbz;
        c2 ^= (c1 ^ ax ^ az ^ bx ^ bz ^ xbz) & anti;
        c1 ^= anti;
    }
    __device__ __forceinline__ u32 phase(u32 fa, u32 fb) const {
        return (fa + fb + (u32)__popcll(c1) + 2u * ((u32)__popcll(c2) & 1u)) & 3u;
    }
};

// Anticommutation parity, PauliStringCore.h:126-146.
__device__ __forceinline__ u64 anti_word(u64 ax, u64 az, u64 bx, u64 bz) {
    return (ax & bz) ^ (az & bx);
}

// Exact FP64 helpers: the reference rounds every product and sum once, so
// the kernels must never contract a multiply into an add.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }

// Host-side launch helpers.
inline int grid_for(i64 n, int per_block, int max_blocks = 1 << 30) {
    i64 g = (n + per_block - 1) / per_block;
    if (g < 1) g = 1;
    if (g > max_blocks) g = max_blocks;
    return (int)g;
}

int sm_count();

}  // namespace pl

// AS dispatch: instantiate a templated body for AS = 1..16 (variadic so
// that commas inside the body survive the preprocessor).
#define PL_AS_CASE(N, ...) \
    case N: {              \
        constexpr int AS = N; \
        __VA_ARGS__;       \
    } break;
#define PL_DISPATCH_AS(as, ...)                                                     \
    switch (as) {                                                                   \
        PL_AS_CASE(1, __VA_ARGS__) PL_AS_CASE(2, __VA_ARGS__) PL_AS_CASE(3, __VA_ARGS__)    \
        PL_AS_CASE(4, __VA_ARGS__) PL_AS_CASE(5, __VA_ARGS__) PL_AS_CASE(6, __VA_ARGS__)    \
        PL_AS_CASE(7, __VA_ARGS__) PL_AS_CASE(8, __VA_ARGS__) PL_AS_CASE(9, __VA_ARGS__)    \
        PL_AS_CASE(10, __VA_ARGS__) PL_AS_CASE(11, __VA_ARGS__) PL_AS_CASE(12, __VA_ARGS__) \
        PL_AS_CASE(13, __VA_ARGS__) PL_AS_CASE(14, __VA_ARGS__) PL_AS_CASE(15, __VA_ARGS__) \
        PL_AS_CASE(16, __VA_ARGS__)                                                 \
        default: return pl::record_status(PL_ERR_INVALID_ARG, "array_size must be 1..16"); \
    }

#define PL_CUDA_TRY(expr)                                 \
    do {                                                  \
        cudaError_t _e = (expr);                          \
        if (_e != cudaSuccess) return pl::record_cuda(_e); \
    } while (0)

namespace pl {
int record_cuda(cudaError_t e);
int record_status(int code, const char* what);
// Measurement hooks (pl_profile_*): launch counter and event-timed passes.
// Process-wide tuning values set through pl_set_tuning (0 = default).
long long tuning(int key);
void note_launch();
// Stream-ordered device allocation from the device's default memory pool
// (freed blocks stay cached in the pool, so regrowing costs no device-wide
// synchronisation and no fresh page mapping); calls are serialised with CUDA
// graph capture on other threads.
cudaError_t dev_alloc(void** p, size_t bytes, cudaStream_t st);
void dev_free(void* p, cudaStream_t st);
void capture_lock();
void capture_unlock();
void note_launches(unsigned long long n);
bool timing_enabled();
void timed_push(cudaEvent_t start, cudaEvent_t stop, unsigned long long bytes, const char* name);
// Small device-to-host reads (output counts, status words, key masks) that
// must not wait behind large copies the caller has queued on other streams:
// a one-warp kernel copies the words into a per-thread pinned, mapped host
// buffer and only this stream is synchronised -- no copy engine is used.
// Each request: `bytes` (a multiple of 4) from a 4-byte aligned device
// address.
struct ReadReq {
    void* host;
    const void* dev;
    size_t bytes;
};
cudaError_t readback_sync(const ReadReq* reqs, int n, cudaStream_t st);
// Fill `bytes` (a multiple of 4, 4-byte aligned) with a 32-bit pattern by a
// kernel: a cudaMemsetAsync may run on a copy engine and then waits behind
// copies the caller has queued on other streams.
cudaError_t fill32_async(void* p, unsigned int value, size_t bytes, cudaStream_t st);
// Several such fills in one launch (at most kMaxFills regions).
struct FillReq {
    void* p;
    unsigned int value;
    size_t bytes;
};
constexpr int kMaxFills = 8;
cudaError_t fill32_multi(const FillReq* reqs, int n, cudaStream_t st);
// Event pair around one launch when timing is enabled (no-op otherwise).
cudaEvent_t timed_begin(cudaStream_t st);
void timed_end(cudaEvent_t start, cudaStream_t st, const char* name, unsigned long long bytes);
}  // namespace pl
