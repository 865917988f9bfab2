// pl_terms.cu -- per-term and per-pair kernels: outer product, commutator,
// apply_CNOT, zero_state_expectation.
//
//   outer product     PauliSum::multiply(rhs), PauliSumOperations.h:256-306;
//                     reference GPU kernel src/gpu/gpu_mul.cu:50-97
//   commutator        commutator_impl, PauliSumOperations.h:316-346;
//                     reference GPU kernel src/gpu/gpu_commutator.cu:25-87
//   apply_CNOT        PauliSumClifford.h:213-239
//   zero_state_exp.   PauliSumUtils.h:163-177

#include <algorithm>
#include <mutex>
#include <vector>

#include "pl_common.cuh"

namespace pl {
namespace {

// ---------------------------------------------------------------------------
// Outer product: out[i*n + j] = lhs[j] * rhs[i].  One CTA row per rhs term
// (held in registers), lhs streamed with coalesced loads (it stays in L2),
// output written with streaming stores -- the kernel is HBM-write bound.
// ---------------------------------------------------------------------------
template <int AS>
__global__ void __launch_bounds__(256)
    k_multiply(const u64* __restrict__ ax, const u64* __restrict__ az, const u8* __restrict__ af,
               const double* __restrict__ av, u64 n, u64 sa, const u64* __restrict__ bx,
               const u64* __restrict__ bz, const u8* __restrict__ bf,
               const double* __restrict__ bv, u64 m, u64 sb, u64* __restrict__ ox,
               u64* __restrict__ oz, u8* __restrict__ of, double* __restrict__ ov, u64 so) {
    for (u64 i = blockIdx.y; i < m; i += gridDim.y) {
        u64 rx[AS], rz[AS];
#pragma unroll
        for (int k = 0; k < AS; ++k) {
            rx[k] = __ldg(bx + k * sb + i);
            rz[k] = __ldg(bz + k * sb + i);
        }
        const u32 rf = __ldg(bf + i);
        const double rv = __ldg(bv + i);
        const u64 row = i * n;
        for (u64 j = (u64)blockIdx.x * blockDim.x + threadIdx.x; j < n;
             j += (u64)gridDim.x * blockDim.x) {
            PhaseAcc acc;
#pragma unroll
            for (int k = 0; k < AS; ++k) {
                const u64 lx = __ldg(ax + k * sa + j), lz = __ldg(az + k * sa + j);
                __stcs(ox + k * so + row + j, lx ^ rx[k]);
                __stcs(oz + k * so + row + j, lz ^ rz[k]);
                acc.step(lx, lz, rx[k], rz[k]);
            }
            __stcs(of + row + j, (u8)acc.phase(__ldg(af + j), rf));
            __stcs(ov + row + j, dmul(__ldg(av + j), rv));
        }
    }
}

// ---------------------------------------------------------------------------
// Commutator with deterministic emission order.
// Pair p = i*m + j (i over lhs, j over rhs), the order of the single-threaded
// CPU commutator_impl.  A tile is 8192 consecutive pairs; each warp tests 32
// consecutive pairs per step (coalesced rhs loads, broadcast lhs loads),
// records the anticommuting ones in shared memory in pair order, and a
// decoupled look-back over tiles turns tile counts into output slots.
// ---------------------------------------------------------------------------
constexpr int kCThreads = 256;
constexpr int kCItems = 32;
constexpr int kCWarpSpan = kCItems * 32;
constexpr u64 kCTile = (u64)kCThreads * kCItems;
constexpr u64 kFlag64Agg = 1ull << 62;
constexpr u64 kFlag64Pre = 2ull << 62;
constexpr u64 kCount64Mask = (1ull << 62) - 1;

__device__ __forceinline__ u64 lookback64(u64* lb, u32 tile, u64 cnt, u64 init, int* status) {
    if (tile == 0) {
        st_volatile64(lb, kFlag64Pre | ((init + cnt) & kCount64Mask));
        return init;
    }
    st_volatile64(lb + tile, kFlag64Agg | cnt);
    u64 excl = 0;
    i64 t = (i64)tile - 1;
    u32 spins = 0;
    while (t >= 0) {
        const u64 w = ld_volatile64(lb + t);
        const u64 fl = w >> 62;
        if (fl == 0) {
            if (++spins > g_spin_limit) {
                raise_status(status, PL_ERR_TIMEOUT);
                break;
            }
            if (spins > 64) __nanosleep(64);
            continue;
        }
        excl += w & kCount64Mask;
        if (fl == 2) break;
        --t;
    }
    st_volatile64(lb + tile, kFlag64Pre | ((excl + cnt) & kCount64Mask));
    return excl;
}

template <int AS>
__global__ void __launch_bounds__(kCThreads)
    k_commutator(const u64* __restrict__ ax, const u64* __restrict__ az,
                 const u8* __restrict__ af, const double* __restrict__ av, u64 n, u64 sa,
                 const u64* __restrict__ bx, const u64* __restrict__ bz,
                 const u8* __restrict__ bf, const double* __restrict__ bv, u64 m, u64 sb,
                 int mul_i,
                 u64* __restrict__ ox, u64* __restrict__ oz, u8* __restrict__ of,
                 double* __restrict__ ov, i64 capacity, unsigned long long* d_count, u64 npairs,
                 u64* lb, u32* tile_ctr, int* status) {
    __shared__ u16 s_emit[kCThreads / 32][kCWarpSpan];
    __shared__ u32 s_wcount[kCThreads / 32];
    __shared__ u32 s_tile;
    __shared__ u64 s_base;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const u32 tile = s_tile;
    const u64 wbase = (u64)tile * kCTile + (u64)warp * kCWarpSpan;
    const u64 p0 = wbase + lane;
    u64 i = p0 / m, j = p0 - (p0 / m) * m;
    u32 cnt = 0;
    for (int t = 0; t < kCItems; ++t) {
        const u64 p = wbase + (u64)t * 32 + lane;
        bool anti = false;
        if (p < npairs) {
            u64 par = 0;
#pragma unroll
            for (int k = 0; k < AS; ++k)
                par ^= anti_word(__ldg(ax + k * sa + i), __ldg(az + k * sa + i),
                                 __ldg(bx + k * sb + j), __ldg(bz + k * sb + j));
            anti = (__popcll(par) & 1) != 0;
        }
        const u32 bal = __ballot_sync(0xffffffffu, anti);
        if (anti) s_emit[warp][cnt + __popc(bal & lanemask_lt())] = (u16)(t * 32 + lane);
        cnt += __popc(bal);
        j += 32;
        while (j >= m && i < n) {
            j -= m;
            ++i;
        }
    }
    if (lane == 0) s_wcount[warp] = cnt;
    __syncthreads();
    if (tid == 0) {
        u64 tot = 0;
        for (int w = 0; w < kCThreads / 32; ++w) tot += s_wcount[w];
        const u64 init = tile == 0 ? (u64)*d_count : 0ull;
        s_base = lookback64(lb, tile, tot, init, status);
        if (tile == gridDim.x - 1) *d_count = (unsigned long long)(s_base + tot);
    }
    __syncthreads();
    u64 wpre = 0;
    for (int w = 0; w < warp; ++w) wpre += s_wcount[w];
    const u64 base = s_base + wpre;
    for (u32 e = lane; e < cnt; e += 32) {
        const u64 p = wbase + s_emit[warp][e];
        const u64 ii = p / m, jj = p - ii * m;
        const i64 slot = (i64)(base + e);
        if (slot >= capacity) {
            raise_status(status, PL_ERR_CAPACITY);
            continue;
        }
        PhaseAcc acc;
#pragma unroll
        for (int k = 0; k < AS; ++k) {
            const u64 lx = __ldg(ax + k * sa + ii), lz = __ldg(az + k * sa + ii);
            const u64 rx = __ldg(bx + k * sb + jj), rz = __ldg(bz + k * sb + jj);
            ox[(i64)k * capacity + slot] = lx ^ rx;
            oz[(i64)k * capacity + slot] = lz ^ rz;
            acc.step(lx, lz, rx, rz);
        }
        of[slot] = (u8)((acc.phase(__ldg(af + ii), __ldg(bf + jj)) + (u32)mul_i) & 3u);
        ov[slot] = dmul(dmul(2.0, __ldg(av + ii)), __ldg(bv + jj));
    }
}

// ---------------------------------------------------------------------------
// Commutator in two passes, for large n*m.  Pass 1 (k_comm_mask): a CTA
// holds 256 rhs terms in registers (one per thread) and streams a tile of
// lhs terms from shared memory (every lane reads the same word: a
// broadcast); each warp's ballot is the anticommutation mask of one lhs
// term against its 32 rhs terms, stored as word (i, j / 32) of a row-major
// bitmask -- pair order i*m + j is the bitmask's bit order.  Pass 2
// (k_comm_emit): tiles of mask words in order, per-tile popcounts, a
// decoupled look-back for the output offsets, and each set bit emitted as
// 2 * lhs_i * rhs_j -- the same terms in the same order as k_commutator.
// The operands are read from L2 once per (lhs tile, rhs tile) instead of
// once per pair.
// ---------------------------------------------------------------------------
constexpr int kMThreads = 256;  // rhs terms per CTA of the mask pass
constexpr int kMLhs = 128;      // lhs terms per CTA of the mask pass
constexpr int kEWords = 8;      // mask words per thread of the emit pass
constexpr u64 kETileW = (u64)kMThreads * kEWords;

template <int AS>
__global__ void __launch_bounds__(kMThreads)
    k_comm_mask(const u64* __restrict__ ax, const u64* __restrict__ az, u64 n, u64 sa,
                const u64* __restrict__ bx, const u64* __restrict__ bz, u64 m, u64 sb,
                u32* __restrict__ mask, u64 mw) {
    __shared__ u64 sx[AS][kMLhs], sz[AS][kMLhs];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const u64 j = (u64)blockIdx.x * kMThreads + tid;
    const u64 i0 = (u64)blockIdx.y * kMLhs;
    const u64 ni = n - i0 < (u64)kMLhs ? n - i0 : (u64)kMLhs;
    for (int t = tid; t < (int)ni * AS; t += kMThreads) {
        const int k = t / (int)ni, r = t - k * (int)ni;
        sx[k][r] = __ldg(ax + (u64)k * sa + i0 + r);
        sz[k][r] = __ldg(az + (u64)k * sa + i0 + r);
    }
    u64 rx[AS], rz[AS];
#pragma unroll
    for (int k = 0; k < AS; ++k) {
        rx[k] = j < m ? __ldg(bx + (u64)k * sb + j) : 0ull;
        rz[k] = j < m ? __ldg(bz + (u64)k * sb + j) : 0ull;
    }
    __syncthreads();
    const u64 w = (u64)blockIdx.x * (kMThreads / 32) + warp;
    if (w >= mw) return;
    u32* row = mask + i0 * mw + w;
#pragma unroll 4
    for (int r = 0; r < (int)ni; ++r) {
        u64 par = 0;
#pragma unroll
        for (int k = 0; k < AS; ++k) par ^= anti_word(sx[k][r], sz[k][r], rx[k], rz[k]);
        const bool anti = j < m && (__popcll(par) & 1);
        const u32 bal = __ballot_sync(0xffffffffu, anti);
        if (lane == 0) row[(u64)r * mw] = bal;
    }
}

template <int AS>
__global__ void __launch_bounds__(kMThreads)
    k_comm_emit(const u64* __restrict__ ax, const u64* __restrict__ az,
                const u8* __restrict__ af, const double* __restrict__ av, u64 sa,
                const u64* __restrict__ bx, const u64* __restrict__ bz,
                const u8* __restrict__ bf, const double* __restrict__ bv, u64 sb, u64 m,
                const u32* __restrict__ mask, u64 nwords, u64 mw, int mul_i,
                u64* __restrict__ ox, u64* __restrict__ oz, u8* __restrict__ of,
                double* __restrict__ ov, i64 capacity, unsigned long long* d_count, u64* lb,
                u32* tile_ctr, int* status) {
    __shared__ u32 s_warp[kMThreads / 32];
    __shared__ u32 s_tile;
    __shared__ u64 s_base;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const u32 tile = s_tile;
    const u64 w0 = (u64)tile * kETileW + (u64)tid * kEWords;
    u32 words[kEWords];
    u32 cnt = 0;
#pragma unroll
    for (int e = 0; e < kEWords; ++e) {
        words[e] = w0 + e < nwords ? __ldg(mask + w0 + e) : 0u;
        cnt += __popc(words[e]);
    }
    u32 inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const u32 t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    u32 wpre = 0, tot = 0;
#pragma unroll
    for (int q = 0; q < kMThreads / 32; ++q) {
        const u32 c = s_warp[q];
        if (q < warp) wpre += c;
        tot += c;
    }
    if (tid == 0) {
        const u64 init = tile == 0 ? (u64)*d_count : 0ull;
        s_base = lookback64(lb, tile, tot, init, status);
        if (tile == gridDim.x - 1) *d_count = (unsigned long long)(s_base + tot);
    }
    __syncthreads();
    u64 slot = s_base + wpre + (inc - cnt);
#pragma unroll
    for (int e = 0; e < kEWords; ++e) {
        u32 bits = words[e];
        if (!bits) continue;
        const u64 wi = w0 + e;
        const u64 i = wi / mw;
        const u64 jb = (wi - i * mw) * 32;
        while (bits) {
            const int b = __ffs(bits) - 1;
            bits &= bits - 1;
            const u64 j = jb + (u64)b;
            if ((i64)slot >= capacity) {
                raise_status(status, PL_ERR_CAPACITY);
                ++slot;
                continue;
            }
            PhaseAcc acc;
#pragma unroll
            for (int k = 0; k < AS; ++k) {
                const u64 lx = __ldg(ax + k * sa + i), lz = __ldg(az + k * sa + i);
                const u64 rx = __ldg(bx + k * sb + j), rz = __ldg(bz + k * sb + j);
                ox[(i64)k * capacity + (i64)slot] = lx ^ rx;
                oz[(i64)k * capacity + (i64)slot] = lz ^ rz;
                acc.step(lx, lz, rx, rz);
            }
            of[slot] = (u8)((acc.phase(__ldg(af + i), __ldg(bf + j)) + (u32)mul_i) & 3u);
            ov[slot] = dmul(dmul(2.0, __ldg(av + i)), __ldg(bv + j));
            ++slot;
        }
    }
    (void)m;
}

// A look-back wait whose predecessor never publishes: tile 1 polls tile 0's
// word, which nothing sets, until the spin limit runs out.
__global__ void k_wait_check(u64* lb, int* status) {
    if (threadIdx.x == 0) (void)lookback64(lb, 1u, 1ull, 0ull, status);
}

// ---------------------------------------------------------------------------
// apply_CNOT: flags ^= (xc & zt & (1 ^ xt ^ zc)) << 1; x_t ^= x_c; z_c ^= z_t.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_cnot(u64* x, u64* z, u8* f, u64 n, u64 stride, int wc,
                                              u64 mc, int wt, u64 mt) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (u64)gridDim.x * blockDim.x) {
        u64* xc_p = x + (u64)wc * stride + i;
        u64* zc_p = z + (u64)wc * stride + i;
        u64* xt_p = x + (u64)wt * stride + i;
        u64* zt_p = z + (u64)wt * stride + i;
        const u64 xc = (*xc_p & mc) != 0, zc = (*zc_p & mc) != 0;
        const u64 xt = (*xt_p & mt) != 0, zt = (*zt_p & mt) != 0;
        f[i] ^= (u8)((xc & zt & (1ull ^ xt ^ zc)) << 1);
        *xt_p ^= (0ull - xc) & mt;
        *zc_p ^= (0ull - zt) & mc;
    }
}

// ---------------------------------------------------------------------------
// zero_state_expectation: one CTA, each thread sums a strided subsequence
// in order, then a fixed binary tree -- deterministic for a given n.
// ---------------------------------------------------------------------------
// zero_state_expectation (PauliSumUtils.h:163-177) over many CTAs: CTA b
// sums the contiguous range [b*per, (b+1)*per) (each thread a strided
// share in order, then a fixed tree) into partial[b]; k_zero_state_total
// adds the partials in a fixed tree.  The grid depends only on the device,
// so the result is deterministic; its order differs from the reference's
// left-to-right sum (1e-10 absolute is the bar).
constexpr int kZThreads = 256;

__device__ __forceinline__ double block_sum_256(double a, double* s) {
    s[threadIdx.x] = a;
    __syncthreads();
    for (int st = kZThreads / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) s[threadIdx.x] = dadd(s[threadIdx.x], s[threadIdx.x + st]);
        __syncthreads();
    }
    return s[0];
}

template <int AS>
__global__ void __launch_bounds__(kZThreads) k_zero_state(const u64* __restrict__ x,
                                                          const u8* __restrict__ f,
                                                          const double* __restrict__ v, u64 n,
                                                          u64 stride, u64 per, double* partial) {
    __shared__ double s[kZThreads];
    const u64 b0 = (u64)blockIdx.x * per;
    const u64 b1 = b0 + per < n ? b0 + per : n;
    double acc = 0.0;
    for (u64 i = b0 + threadIdx.x; i < b1; i += kZThreads) {
        u64 any = 0;
#pragma unroll
        for (int k = 0; k < AS; ++k) any |= __ldg(x + k * stride + i);
        const u32 fl = __ldg(f + i);
        if (any == 0 && (fl & 1u) == 0) {
            const double val = __ldg(v + i);
            acc = dadd(acc, (fl & 2u) ? -val : val);
        }
    }
    const double t = block_sum_256(acc, s);
    if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

__global__ void __launch_bounds__(kZThreads) k_zero_state_total(const double* partial, int np,
                                                                double* out) {
    __shared__ double s[kZThreads];
    double acc = 0.0;
    for (int i = threadIdx.x; i < np; i += kZThreads) acc = dadd(acc, partial[i]);
    const double t = block_sum_256(acc, s);
    if (threadIdx.x == 0) *out = t;
}

}  // namespace

PL_SPIN_LIMIT_SETTER(set_spin_limit_terms)

// ---------------------------------------------------------------------------
// Host entry points (internal).
// ---------------------------------------------------------------------------
int multiply_impl(int as, const u64* ax, const u64* az, const u8* af, const double* av, i64 n,
                  i64 sa, const u64* bx, const u64* bz, const u8* bf, const double* bv, i64 m,
                  i64 sb, u64* ox, u64* oz, u8* of, double* ov, i64 so, cudaStream_t st) {
    if (as < 1 || as > kMaxAS || n < 0 || m < 0 || (n > 0 && m > (1ll << 40) / n))
        return record_status(PL_ERR_INVALID_ARG, "multiply: bad array_size or size");
    if (n == 0 || m == 0) return record_status(PL_OK, nullptr);
    if (!ax || !az || !af || !av || !bx || !bz || !bf || !bv || !ox || !oz || !of || !ov)
        return record_status(PL_ERR_INVALID_ARG, "multiply: null pointer");
    const dim3 grid((unsigned)grid_for(n, 256, 2048), (unsigned)std::min<i64>(m, 65535));
    PL_DISPATCH_AS(as, k_multiply<AS><<<grid, 256, 0, st>>>(ax, az, af, av, (u64)n, (u64)sa, bx,
                                                           bz, bf, bv, (u64)m, (u64)sb, ox, oz,
                                                           of, ov, (u64)so), pl::note_launch());
    PL_CUDA_TRY(cudaGetLastError());
    return record_status(PL_OK, nullptr);
}

// Scratch for the commutator's tile look-back: one u64 per 8192 pairs plus
// a tile counter and a status word.
size_t commutator_scratch_bytes(u64 npairs) {
    const u64 tiles = (npairs + kCTile - 1) / kCTile;
    return (size_t)tiles * 8 + 256;
}

// The two-pass form needs a bitmask of n * ceil(m/32) words; it is used when
// there are enough pairs to fill the device and the mask stays modest.
constexpr u64 kMaskMaxBytes = 1ull << 30;
bool use_mask_form(u64 n, u64 m) {
    const u64 mw = (m + 31) / 32;
    return n * m >= (1ull << 22) && n * mw * 4 <= kMaskMaxBytes && n <= (1ull << 31) &&
           m <= (1ull << 31);
}
size_t commutator_mask_scratch_bytes(u64 n, u64 m) {
    const u64 mw = (m + 31) / 32;
    const u64 tiles = (n * mw + kETileW - 1) / kETileW;
    return (size_t)(256 + tiles * 8 + 256) + (size_t)(n * mw * 4);
}

int commutator_launch_mask(int as, int mul_i, const u64* ax, const u64* az, const u8* af,
                           const double* av, i64 n, i64 sa, const u64* bx, const u64* bz,
                           const u8* bf, const double* bv, i64 m, i64 sb, u64* ox, u64* oz,
                           u8* of, double* ov, i64 capacity, unsigned long long* d_count,
                           void* scratch, int* d_status, cudaStream_t st) {
    const u64 mw = ((u64)m + 31) / 32;
    const u64 nwords = (u64)n * mw;
    const u64 tiles = (nwords + kETileW - 1) / kETileW;
    unsigned char* s = (unsigned char*)scratch;
    u32* tile_ctr = (u32*)s;
    u64* lb = (u64*)(s + 256);
    u32* mask = (u32*)(s + 256 + tiles * 8 + 256);
    PL_CUDA_TRY(fill32_async(scratch, 0u, 256 + tiles * 8, st));
    const dim3 mgrid((unsigned)((m + kMThreads - 1) / kMThreads),
                     (unsigned)((n + kMLhs - 1) / kMLhs));
    PL_DISPATCH_AS(as, k_comm_mask<AS><<<mgrid, kMThreads, 0, st>>>(
                           ax, az, (u64)n, (u64)sa, bx, bz, (u64)m, (u64)sb, mask, mw),
                   pl::note_launch());
    PL_DISPATCH_AS(as, k_comm_emit<AS><<<(unsigned)tiles, kMThreads, 0, st>>>(
                           ax, az, af, av, (u64)sa, bx, bz, bf, bv, (u64)sb, (u64)m, mask,
                           nwords, mw, mul_i, ox, oz, of, ov, capacity, d_count, lb, tile_ctr,
                           d_status), pl::note_launch());
    PL_CUDA_TRY(cudaGetLastError());
    return PL_OK;
}

int commutator_launch(int as, int mul_i, const u64* ax, const u64* az, const u8* af,
                      const double* av, i64 n, i64 sa, const u64* bx, const u64* bz,
                      const u8* bf, const double* bv, i64 m, i64 sb, u64* ox, u64* oz, u8* of,
                      double* ov, i64 capacity, unsigned long long* d_count, void* scratch,
                      int* d_status, cudaStream_t st) {
    const u64 npairs = (u64)n * (u64)m;
    const u64 tiles = (npairs + kCTile - 1) / kCTile;
    unsigned char* s = (unsigned char*)scratch;
    u64* lb = (u64*)(s + 256);
    u32* tile_ctr = (u32*)s;
    // a fill kernel, not a copy-engine memset: it never queues behind a
    // caller's large copies on other streams
    PL_CUDA_TRY(fill32_async(scratch, 0u, commutator_scratch_bytes(npairs), st));
    PL_DISPATCH_AS(as, k_commutator<AS><<<(unsigned)tiles, kCThreads, 0, st>>>(
                           ax, az, af, av, (u64)n, (u64)sa, bx, bz, bf, bv, (u64)m, (u64)sb,
                           mul_i, ox, oz, of, ov, capacity, d_count, npairs, lb, tile_ctr,
                           d_status), pl::note_launch());
    PL_CUDA_TRY(cudaGetLastError());
    return PL_OK;
}

// The commutator with stream-ordered scratch.  With `wait` the call reads the
// device status back (a stream synchronisation) and reports a capacity or
// look-back failure; without it the call is asynchronous like the
// reference's launcher (paulib_gpu_api.h:35-42): nothing waits on the host,
// the scratch is released in stream order, and an output that did not fit
// shows as *d_count > capacity.
int commutator_impl(int as, int mul_i, const u64* ax, const u64* az, const u8* af,
                    const double* av, i64 n, i64 sa, const u64* bx, const u64* bz, const u8* bf,
                    const double* bv, i64 m, i64 sb, u64* ox, u64* oz, u8* of, double* ov,
                    i64 capacity, unsigned long long* d_count, bool wait, cudaStream_t st) {
    if (as < 1 || as > kMaxAS || n < 0 || m < 0 || capacity < 0 || !d_count ||
        (n > 0 && m > (1ll << 40) / n))
        return record_status(PL_ERR_INVALID_ARG, "commutator: bad array_size or size");
    if (n == 0 || m == 0) return record_status(PL_OK, nullptr);
    if (!ax || !az || !af || !av || !bx || !bz || !bf || !bv || !ox || !oz || !of || !ov)
        return record_status(PL_ERR_INVALID_ARG, "commutator: null pointer");
    // Stream-ordered scratch: safe when several streams call concurrently.
    const bool two_pass = use_mask_form((u64)n, (u64)m);
    const size_t bytes = (two_pass ? commutator_mask_scratch_bytes((u64)n, (u64)m)
                                   : commutator_scratch_bytes((u64)n * (u64)m)) + 256;
    void* scratch = nullptr;
    // from the device pool with its cached blocks kept (dev_alloc): a call
    // then maps no fresh memory
    if (dev_alloc(&scratch, bytes, st) != cudaSuccess) {
        cudaGetLastError();
        return record_status(PL_ERR_OOM, "commutator scratch");
    }
    int* d_status = (int*)((unsigned char*)scratch + bytes - 256);
    int rc = PL_OK;
    cudaError_t e = fill32_async(d_status, 0u, sizeof(int), st);
    if (e != cudaSuccess) rc = record_cuda(e);
    if (rc == PL_OK && two_pass)
        rc = commutator_launch_mask(as, mul_i, ax, az, af, av, n, sa, bx, bz, bf, bv, m, sb, ox,
                                    oz, of, ov, capacity, d_count, scratch, d_status, st);
    else if (rc == PL_OK)
        rc = commutator_launch(as, mul_i, ax, az, af, av, n, sa, bx, bz, bf, bv, m, sb, ox, oz,
                               of, ov, capacity, d_count, scratch, d_status, st);
    int dstat = 0;
    if (rc == PL_OK && wait) {
        // the capacity / timeout check needs the device status
        const ReadReq rr[1] = {{&dstat, d_status, sizeof(int)}};
        e = readback_sync(rr, 1, st);
        if (e != cudaSuccess) rc = record_cuda(e);
    }
    dev_free(scratch, st);
    if (rc != PL_OK) return rc;
    if (dstat != 0) return record_status(dstat, "commutator: device-side check");
    return record_status(PL_OK, nullptr);
}

}  // namespace pl

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using namespace pl;

extern "C" void launch_gpu_mul_soa(int array_size, const uint64_t* lhs_x, const uint64_t* lhs_z,
                                   const uint8_t* lhs_flags, const double* lhs_val,
                                   const uint64_t* rhs_x, const uint64_t* rhs_z,
                                   const uint8_t* rhs_flags, const double* rhs_val,
                                   uint64_t* out_x, uint64_t* out_z, uint8_t* out_flags,
                                   double* out_val, int n, int m, cudaStream_t stream) {
    multiply_impl(array_size, (const u64*)lhs_x, (const u64*)lhs_z, lhs_flags, lhs_val, n, n,
                  (const u64*)rhs_x, (const u64*)rhs_z, rhs_flags, rhs_val, m, m, (u64*)out_x,
                  (u64*)out_z, out_flags, out_val, (i64)n * m, stream);
}

extern "C" int pl_multiply(int array_size, const uint64_t* lhs_x, const uint64_t* lhs_z,
                           const uint8_t* lhs_flags, const double* lhs_val, int64_t n,
                           const uint64_t* rhs_x, const uint64_t* rhs_z,
                           const uint8_t* rhs_flags, const double* rhs_val, int64_t m,
                           uint64_t* out_x, uint64_t* out_z, uint8_t* out_flags, double* out_val,
                           cudaStream_t stream) {
    return multiply_impl(array_size, (const u64*)lhs_x, (const u64*)lhs_z, lhs_flags, lhs_val, n,
                         n, (const u64*)rhs_x, (const u64*)rhs_z, rhs_flags, rhs_val, m, m,
                         (u64*)out_x, (u64*)out_z, out_flags, out_val, n * m, stream);
}

extern "C" void launch_gpu_commutator_soa(int array_size, int multiply_by_i,
                                          const uint64_t* lhs_x, const uint64_t* lhs_z,
                                          const uint8_t* lhs_flags, const double* lhs_val,
                                          const uint64_t* rhs_x, const uint64_t* rhs_z,
                                          const uint8_t* rhs_flags, const double* rhs_val,
                                          uint64_t* out_x, uint64_t* out_z, uint8_t* out_flags,
                                          double* out_val, unsigned long long* d_count, int n,
                                          int m, long long capacity, cudaStream_t stream) {
    commutator_impl(array_size, multiply_by_i ? 1 : 0, (const u64*)lhs_x, (const u64*)lhs_z,
                    lhs_flags, lhs_val, n, n, (const u64*)rhs_x, (const u64*)rhs_z, rhs_flags,
                    rhs_val, m, m, (u64*)out_x, (u64*)out_z, out_flags, out_val, capacity,
                    d_count, false, stream);
}

extern "C" int pl_commutator(int array_size, int multiply_by_i, const uint64_t* lhs_x,
                             const uint64_t* lhs_z, const uint8_t* lhs_flags,
                             const double* lhs_val, int64_t n, const uint64_t* rhs_x,
                             const uint64_t* rhs_z, const uint8_t* rhs_flags,
                             const double* rhs_val, int64_t m, uint64_t* out_x, uint64_t* out_z,
                             uint8_t* out_flags, double* out_val, int64_t capacity,
                             unsigned long long* d_count, cudaStream_t stream) {
    return commutator_impl(array_size, multiply_by_i ? 1 : 0, (const u64*)lhs_x,
                           (const u64*)lhs_z, lhs_flags, lhs_val, n, n, (const u64*)rhs_x,
                           (const u64*)rhs_z, rhs_flags, rhs_val, m, m, (u64*)out_x,
                           (u64*)out_z, out_flags, out_val, capacity, d_count, true, stream);
}

extern "C" int pl_check_bounded_wait(int* device_status) {
    if (!device_status) return record_status(PL_ERR_INVALID_ARG, "pl_check_bounded_wait");
    void* p = nullptr;
    PL_CUDA_TRY(cudaMalloc(&p, 256));
    u64* lb = static_cast<u64*>(p);
    int* status = reinterpret_cast<int*>(static_cast<unsigned char*>(p) + 128);
    cudaError_t e = cudaMemset(p, 0, 256);
    if (e == cudaSuccess) {
        k_wait_check<<<1, 32>>>(lb, status);
        note_launch();
        e = cudaGetLastError();
    }
    int st = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&st, status, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(p);
    if (e != cudaSuccess) return record_cuda(e);
    *device_status = st;
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_apply_cnot(int array_size, uint64_t* x, uint64_t* z, uint8_t* flags, int64_t n,
                             int64_t stride, int control, int target, cudaStream_t stream) {
    if (array_size < 1 || array_size > kMaxAS || n < 0 || stride < n || control < 0 ||
        target < 0 || control >= 64 * array_size || target >= 64 * array_size ||
        control == target)
        return record_status(PL_ERR_INVALID_ARG, "pl_apply_cnot: bad argument");
    if (n == 0) return record_status(PL_OK, nullptr);
    if (!x || !z || !flags) return record_status(PL_ERR_INVALID_ARG, "pl_apply_cnot: null");
    k_cnot<<<grid_for(n, 256, sm_count() * 8), 256, 0, stream>>>(
        (u64*)x, (u64*)z, flags, (u64)n, (u64)stride, control / 64, 1ull << (control % 64),
        target / 64, 1ull << (target % 64)), pl::note_launch();
    PL_CUDA_TRY(cudaGetLastError());
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_zero_state_expectation(int array_size, const uint64_t* x, const uint8_t* flags,
                                         const double* val, int64_t n, int64_t stride,
                                         double* d_result, cudaStream_t stream) {
    if (array_size < 1 || array_size > kMaxAS || n < 0 || stride < n || !d_result)
        return record_status(PL_ERR_INVALID_ARG, "pl_zero_state_expectation: bad argument");
    if (n > 0 && (!x || !flags || !val))
        return record_status(PL_ERR_INVALID_ARG, "pl_zero_state_expectation: null");
    // one partial per CTA, in stream-ordered scratch from the device pool
    const int nb = std::max(1, std::min(2 * sm_count(), (int)((n + kZThreads - 1) / kZThreads)));
    const u64 per = ((u64)n + nb - 1) / (u64)nb;
    void* scratch = nullptr;
    if (dev_alloc(&scratch, sizeof(double) * (size_t)nb, stream) != cudaSuccess) {
        cudaGetLastError();
        return record_status(PL_ERR_OOM, "zero_state_expectation scratch");
    }
    double* partial = static_cast<double*>(scratch);
    PL_DISPATCH_AS(array_size, k_zero_state<AS><<<nb, kZThreads, 0, stream>>>(
                                   (const u64*)x, flags, val, (u64)n, (u64)stride, per, partial),
                   pl::note_launch());
    k_zero_state_total<<<1, kZThreads, 0, stream>>>(partial, nb, d_result), pl::note_launch();
    const cudaError_t e = cudaGetLastError();
    dev_free(scratch, stream);
    PL_CUDA_TRY(e);
    return record_status(PL_OK, nullptr);
}

// ---------------------------------------------------------------------------
// Commutator without allocation.
//
// Some callers cannot let a library allocate device memory: hosts that carve
// the whole device into their own pool up front (an HBM-budgeted serving
// process, a framework with its own caching allocator), and callers that
// cannot afford the device-wide synchronisation that cudaMalloc / cudaFree
// may cause.  pl_commutator_noalloc runs the same kernel as pl_commutator
// but keeps its only scratch -- the per-tile look-back words, the tile
// counter and the status word -- in the file-scope array below, which every
// GPU that loads this library holds until the process exits.
// ---------------------------------------------------------------------------
namespace pl {
namespace {
constexpr u64 kNoAllocMaxTiles = 1ull << 16;  // 2^16 tiles of 8192 pairs = 2^29 pairs
constexpr size_t kNoAllocBytes = 256 + kNoAllocMaxTiles * 8 + 256;
static __device__ __align__(256) unsigned char g_commutator_scratch[kNoAllocBytes];

// Device address of g_commutator_scratch, looked up once per device with
// that device current.  In host code the symbol is only a host-side stand-in,
// so the kernel must be given this address instead.
int noalloc_scratch(void** ptr) {
    static std::mutex mu;
    static std::vector<void*> by_device;
    int dev = 0;
    PL_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if ((int)by_device.size() <= dev) by_device.resize(dev + 1, nullptr);
    if (!by_device[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_commutator_scratch);
        if (e != cudaSuccess) return record_cuda(e);
        by_device[dev] = p;
    }
    *ptr = by_device[dev];
    return PL_OK;
}
}  // namespace
}  // namespace pl

extern "C" int pl_commutator_noalloc(int array_size, int multiply_by_i, const uint64_t* lhs_x,
                                     const uint64_t* lhs_z, const uint8_t* lhs_flags,
                                     const double* lhs_val, int64_t n, const uint64_t* rhs_x,
                                     const uint64_t* rhs_z, const uint8_t* rhs_flags,
                                     const double* rhs_val, int64_t m, uint64_t* out_x,
                                     uint64_t* out_z, uint8_t* out_flags, double* out_val,
                                     int64_t capacity, unsigned long long* d_count,
                                     cudaStream_t stream) {
    if (array_size < 1 || array_size > kMaxAS || n < 0 || m < 0 || capacity < 0 || !d_count)
        return record_status(PL_ERR_INVALID_ARG, "pl_commutator_noalloc: bad argument");
    if (n == 0 || m == 0) return record_status(PL_OK, nullptr);
    const u64 npairs = (u64)n * (u64)m;
    if ((u64)m > (kNoAllocMaxTiles * kCTile) / (u64)n)
        return record_status(PL_ERR_INVALID_ARG,
                             "pl_commutator_noalloc: n*m exceeds the 2^29-pair limit of its "
                             "static scratch (use pl_commutator)");
    if (!lhs_x || !lhs_z || !lhs_flags || !lhs_val || !rhs_x || !rhs_z || !rhs_flags ||
        !rhs_val || !out_x || !out_z || !out_flags || !out_val)
        return record_status(PL_ERR_INVALID_ARG, "pl_commutator_noalloc: null pointer");
    void* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    int* d_status = (int*)((unsigned char*)scratch + kNoAllocBytes - 256);
    // the array keeps the previous call's contents: clear what must start at 0
    // (a fill kernel; the look-back words are cleared by commutator_launch)
    PL_CUDA_TRY(fill32_async(d_status, 0u, sizeof(int), stream));
    rc = commutator_launch(array_size, multiply_by_i ? 1 : 0, (const u64*)lhs_x,
                           (const u64*)lhs_z, lhs_flags, lhs_val, n, n, (const u64*)rhs_x,
                           (const u64*)rhs_z, rhs_flags, rhs_val, m, m, (u64*)out_x,
                           (u64*)out_z, out_flags, out_val, capacity, d_count, scratch, d_status,
                           stream);
    if (rc) return rc;
    (void)npairs;
    // The 4-byte status comes back by a plain copy into this stack variable:
    // the mapped pinned buffer the other entry points read through is
    // allocated on a thread's first use, which this entry point must not do.
    int dstat = 0;
    PL_CUDA_TRY(cudaMemcpyAsync(&dstat, d_status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    PL_CUDA_TRY(cudaStreamSynchronize(stream));
    if (dstat != 0) return record_status(dstat, "pl_commutator_noalloc: device-side check");
    return record_status(PL_OK, nullptr);
}
