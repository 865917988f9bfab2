// pl_shard.cu -- the device half of the hash-owned sharded collate
// (MpiPauliSum.h:101-181): every term belongs to rank owner = FNV-1a(x, z)
// mod ranks (the phase is excluded, so P, -P and iP meet on one rank).  A
// rank packs its terms into per-owner buckets, the buckets travel with one
// all-to-all (NCCL over NVLink, driven from the host), and the receiver
// unpacks them and canonicalizes locally; the union of the ranks' results is
// the canonical global sum.
//
// Records are term-major u64 words: x[0..AS), z[0..AS), flags, the value's
// bits -- one contiguous buffer per rank, so the exchange is one
// all-to-all of a single dtype.  Buckets keep the terms' order (stable), as
// the reference's packing loop does.

#include "pl_common.cuh"

namespace pl {
int state_planes(pl_state* s, u64** x, u64** z, u8** f, double** v, i64* cap, i64* n);
int state_reserve(pl_state* s, i64 n);
int state_set_size(pl_state* s, i64 n);
cudaStream_t state_stream(pl_state* s);
int state_array_size(pl_state* s);

namespace {

constexpr int kShardThreads = 256;
constexpr int kShardItems = 8;
constexpr int kShardTile = kShardThreads * kShardItems;  // 2048 terms
constexpr int kMaxRanks = 64;

struct Planes {
    const u64* x;
    const u64* z;
    const u8* f;
    const double* v;
    i64 cap;
};

// pattern_hash (MpiPauliSum.h:72-80): FNV-1a over x[k], z[k] alternating.
template <int AS>
__device__ __forceinline__ u32 owner_of(const Planes& P, i64 i, u32 ranks) {
    u64 h = 0xcbf29ce484222325ull;
#pragma unroll
    for (int k = 0; k < AS; ++k) {
        h = (h ^ P.x[k * P.cap + i]) * 0x100000001b3ull;
        h = (h ^ P.z[k * P.cap + i]) * 0x100000001b3ull;
    }
    return (u32)(h % ranks);
}

// Per tile and owner: how many of the tile's terms go there; each term's
// owner is kept for the scatter.
template <int AS>
__global__ void __launch_bounds__(kShardThreads) k_owner_count(Planes P, i64 n, u32 ranks,
                                                               u8* owner, u32* tile_counts) {
    __shared__ u32 sh[kMaxRanks];
    for (u32 g = threadIdx.x; g < ranks; g += blockDim.x) sh[g] = 0;
    __syncthreads();
    const i64 base = (i64)blockIdx.x * kShardTile;
    for (int t = 0; t < kShardItems; ++t) {
        const i64 i = base + t * kShardThreads + threadIdx.x;
        if (i < n) {
            const u32 o = owner_of<AS>(P, i, ranks);
            owner[i] = (u8)o;
            atomicAdd(&sh[o], 1u);
        }
    }
    __syncthreads();
    for (u32 g = threadIdx.x; g < ranks; g += blockDim.x)
        tile_counts[(size_t)blockIdx.x * ranks + g] = sh[g];
}

// One block per owner: exclusive scan of its tile counts (in place) and its
// total.
__global__ void __launch_bounds__(1024) k_owner_scan(u32* tile_counts, u32 tiles, u32 ranks,
                                                     u64* totals) {
    __shared__ u32 sw[32];
    __shared__ u64 carry;
    const u32 g = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (u32 b0 = 0; b0 < tiles; b0 += 1024) {
        const u32 t = b0 + threadIdx.x;
        const u32 c = t < tiles ? tile_counts[(size_t)t * ranks + g] : 0u;
        u32 inc = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 v = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += v;
        }
        if (lane == 31) sw[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            const u32 w = sw[lane];
            u32 wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const u32 v = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += v;
            }
            sw[lane] = wi - w;
        }
        __syncthreads();
        const u64 ex = carry + sw[warp] + (inc - c);
        if (t < tiles) tile_counts[(size_t)t * ranks + g] = (u32)ex;
        __syncthreads();
        if (threadIdx.x == 1023) carry = ex + c;
        __syncthreads();
    }
    if (threadIdx.x == 0) totals[g] = carry;
}

// Stable scatter of term records into the owners' buckets: a term's place is
// its owner's bucket start + the owner's count in earlier tiles + its rank
// among the tile's terms of that owner (term order).
template <int AS>
__global__ void __launch_bounds__(kShardThreads) k_owner_scatter(Planes P, i64 n, u32 ranks,
                                                                 const u8* owner,
                                                                 const u32* tile_offs,
                                                                 const u64* bucket_start,
                                                                 u64* rec) {
    __shared__ u32 sh[kMaxRanks];
    constexpr int W = 2 * AS + 2;
    for (u32 g = threadIdx.x; g < ranks; g += blockDim.x) sh[g] = 0;
    __syncthreads();
    const i64 base = (i64)blockIdx.x * kShardTile;
    const int lane = threadIdx.x & 31;
    // rows of 256 terms in order; within a row, warp 0's 32 terms first
    for (int t = 0; t < kShardItems; ++t) {
        const i64 i = base + t * kShardThreads + threadIdx.x;
        const bool valid = i < n;
        const u32 o = valid ? owner[i] : 0xffffffffu;
        const u32 peers = __match_any_sync(0xffffffffu, o);
        const u32 before_in_warp = __popc(peers & lanemask_lt());
        // warps of the row in order: a warp's leader claims its run
        u32 run_base = 0;
        for (int w = 0; w < kShardThreads / 32; ++w) {
            if ((int)(threadIdx.x >> 5) == w && valid && lane == __ffs(peers) - 1)
                run_base = atomicAdd(&sh[o], (u32)__popc(peers));
            __syncthreads();
        }
        run_base = __shfl_sync(0xffffffffu, run_base, __ffs(peers) - 1);
        if (valid) {
            const u64 pos =
                bucket_start[o] + tile_offs[(size_t)blockIdx.x * ranks + o] + run_base +
                before_in_warp;
            u64* r = rec + pos * W;
#pragma unroll
            for (int k = 0; k < AS; ++k) {
                r[k] = P.x[k * P.cap + i];
                r[AS + k] = P.z[k * P.cap + i];
            }
            r[2 * AS] = P.f[i];
            r[2 * AS + 1] = (u64)__double_as_longlong(P.v[i]);
        }
    }
}

// Records back into SoA planes, in record order.
template <int AS>
__global__ void __launch_bounds__(256) k_unpack(const u64* rec, i64 n, u64* x, u64* z, u8* f,
                                                double* v, i64 cap) {
    constexpr int W = 2 * AS + 2;
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (i64)gridDim.x * blockDim.x) {
        const u64* r = rec + i * W;
#pragma unroll
        for (int k = 0; k < AS; ++k) {
            x[k * cap + i] = r[k];
            z[k * cap + i] = r[AS + k];
        }
        f[i] = (u8)r[2 * AS];
        v[i] = __longlong_as_double((long long)r[2 * AS + 1]);
    }
}

}  // namespace
}  // namespace pl

using namespace pl;

extern "C" int pl_state_shard_pack(pl_state* s, int ranks, uint64_t* records, int64_t capacity,
                                   int64_t* counts) {
    if (!s || ranks < 1 || ranks > kMaxRanks || !counts)
        return record_status(PL_ERR_INVALID_ARG, "pl_state_shard_pack");
    u64 *x, *z;
    u8* f;
    double* v;
    i64 cap, n;
    int rc = state_planes(s, &x, &z, &f, &v, &cap, &n);
    if (rc) return rc;
    for (int g = 0; g < ranks; ++g) counts[g] = 0;
    if (n == 0) return record_status(PL_OK, nullptr);
    if (!records || capacity < n)
        return record_status(PL_ERR_CAPACITY, "pl_state_shard_pack: record buffer too small");
    const int as = state_array_size(s);
    const cudaStream_t st = state_stream(s);
    const u32 tiles = (u32)((n + kShardTile - 1) / kShardTile);
    // scratch: owners, per-tile counts, totals / bucket starts
    const size_t b_own = ((size_t)n + 255) & ~size_t(255);
    const size_t b_cnt = (((size_t)tiles * ranks * 4) + 255) & ~size_t(255);
    const size_t bytes = b_own + b_cnt + 2 * 8 * kMaxRanks;
    void* mem = nullptr;
    PL_CUDA_TRY(dev_alloc(&mem, bytes, st));
    u8* owner = static_cast<u8*>(mem);
    u32* tile_counts = reinterpret_cast<u32*>(static_cast<unsigned char*>(mem) + b_own);
    u64* totals = reinterpret_cast<u64*>(static_cast<unsigned char*>(mem) + b_own + b_cnt);
    u64* starts = totals + kMaxRanks;
    const Planes P{x, z, f, v, cap};
    PL_DISPATCH_AS(as, k_owner_count<AS><<<tiles, kShardThreads, 0, st>>>(P, n, (u32)ranks, owner,
                                                                          tile_counts),
                   pl::note_launch());
    k_owner_scan<<<ranks, 1024, 0, st>>>(tile_counts, tiles, (u32)ranks, totals),
        pl::note_launch();
    u64 tot[kMaxRanks], start[kMaxRanks];
    PL_CUDA_TRY(cudaMemcpyAsync(tot, totals, 8 * ranks, cudaMemcpyDeviceToHost, st));
    PL_CUDA_TRY(cudaStreamSynchronize(st));
    u64 acc = 0;
    for (int g = 0; g < ranks; ++g) {
        start[g] = acc;
        acc += tot[g];
        counts[g] = (int64_t)tot[g];
    }
    PL_CUDA_TRY(cudaMemcpyAsync(starts, start, 8 * ranks, cudaMemcpyHostToDevice, st));
    PL_DISPATCH_AS(as, k_owner_scatter<AS><<<tiles, kShardThreads, 0, st>>>(
                           P, n, (u32)ranks, owner, tile_counts, starts, (u64*)records),
                   pl::note_launch());
    PL_CUDA_TRY(cudaGetLastError());
    dev_free(mem, st);
    PL_CUDA_TRY(cudaStreamSynchronize(st));
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_state_shard_unpack(pl_state* s, const uint64_t* records, int64_t n) {
    if (!s || n < 0 || (n > 0 && !records) || n >= (1ll << 30))
        return record_status(PL_ERR_INVALID_ARG, "pl_state_shard_unpack");
    int rc = state_reserve(s, n);
    if (rc) return rc;
    u64 *x, *z;
    u8* f;
    double* v;
    i64 cap, cur;
    rc = state_planes(s, &x, &z, &f, &v, &cap, &cur);
    if (rc) return rc;
    const int as = state_array_size(s);
    const cudaStream_t st = state_stream(s);
    if (n > 0)
        PL_DISPATCH_AS(as, k_unpack<AS><<<grid_for(n, 256, sm_count() * 8), 256, 0, st>>>(
                               (const u64*)records, n, x, z, f, v, cap),
                       pl::note_launch());
    PL_CUDA_TRY(cudaGetLastError());
    rc = state_set_size(s, n);
    if (rc) return rc;
    return record_status(PL_OK, nullptr);
}
