// pl_propagate.cu -- device-resident Pauli propagation (evolve + truncate).
//
// Reference semantics (PauLIB):
//   evolve            PauliSumOperations.h:107-183  per rotation (P, theta):
//                     ps = iP; fast paths at theta ~ 0, pi, +-pi/2 (isCloseOne,
//                     eps 1e-14); otherwise anticommuting Q keeps cos*c in place
//                     and appends (Q*ps, -sin*c), then `+=` (sort_and_combine).
//   apply_truncation  PauliPropagation.h:36-47  canonicalize, truncate_weight,
//                     cutoff (trim when max_terms is set).
//   propagate         PauliPropagation.h:54-63  gates in reverse order.
//   apply_CNOT        PauliSumClifford.h:213-239.
//
// Fast path (the state is canonical: sorted by (x, z, phase), sign folded,
// keys distinct; the generator is a single-qubit Pauli).  Per rotation:
//   A  k_expand        anticommutation test; each anticommuting term's child
//                      Q*ps goes to one of two runs by the value of the
//                      flipped bit.  Flipping one bit preserves the order
//                      inside each run (the only local inversion, between
//                      the phase-0 / phase-1 twins of one string, is fixed
//                      in place), so no sort is needed.
//   B  k_merge_runs    merge-path merge of the two runs.
//   C  k_merge_reduce  merge-path merge of the scaled old terms with the
//                      children, segment reduce, zero / weight / cutoff
//                      filter and look-back compaction into the other buffer.
// Every canonical key receives at most one old and one new contribution, so
// the two-stage order of the reference (`+=` then canonicalize) reduces to
// S(sign 0) - S(sign 1) of at most two terms: bit-identical to the reference.
// Overflow of the output buffer is detected on the device; the host replays
// from the failing gate after growing the buffers, so the fast path never
// waits for the host.
//
// Other states and generators take the general path: materialise old and
// new terms, then the collate engine (pl_collate.cu) in the matching mode.

#include <cuda_pipeline.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "pl_budget.h"
#include "pl_collate.cuh"

namespace pl {
namespace {

constexpr int kPT = 256;
constexpr int kExpItems = 8;
constexpr u32 kExpTile = kPT * kExpItems;
constexpr u64 kF2Agg = 1ull << 62, kF2Pre = 2ull << 62;
constexpr u64 kC31 = (1ull << 31) - 1;

template <int AS>
struct PItems {
    static constexpr int v = AS == 1 ? 8 : AS == 2 ? 4 : AS <= 4 ? 2 : 1;
};
template <int AS>
constexpr int ptile() {
    return kPT * PItems<AS>::v;
}

struct Buf {
    u64* x;
    u64* z;
    u8* f;
    double* v;
    i64 cap;
};

enum RotMode : int { kSkip = 0, kNegate = 1, kHalfPos = 2, kHalfNeg = 3, kGeneral = 4 };

template <int AS>
struct GateP {
    u64 px[AS], pz[AS];
    u32 psf;     // flags of ps = P with its phase flipped
    int cw;      // class bit: word,
    u64 cmask;   //            mask,
    int cls_x;   //            and plane (1: x, 0: z)
};

// One op of a propagation as the fast-path kernels read it from device
// memory, so a chain of rotations can be replayed from a CUDA graph.
template <int AS>
struct GateRec {
    GateP<AS> g;
    int mode;
    int op;        // op index (reported on a capacity overflow)
    double c;      // cos(theta)
    double neg_s;  // -sin(theta)
};

__device__ __forceinline__ int status_set(const int* status) {
    return *reinterpret_cast<const volatile int*>(status);
}

// Order key of a term: (x, z, phase, sign); ps = phase << 1 | sign.
__device__ __forceinline__ u32 ps_of(u32 f) { return ((f & 1u) << 1) | ((f >> 1) & 1u); }

template <int AS>
struct Key {
    u64 x[AS], z[AS];
    u32 ps;
};

template <int AS>
__device__ __forceinline__ int kcmp(const Key<AS>& a, const Key<AS>& b) {
#pragma unroll
    for (int k = 0; k < AS; ++k)
        if (a.x[k] != b.x[k]) return a.x[k] < b.x[k] ? -1 : 1;
#pragma unroll
    for (int k = 0; k < AS; ++k)
        if (a.z[k] != b.z[k]) return a.z[k] < b.z[k] ? -1 : 1;
    if (a.ps != b.ps) return a.ps < b.ps ? -1 : 1;
    return 0;
}

template <int AS>
__device__ __forceinline__ Key<AS> gkey(const Buf& B, i64 i) {
    Key<AS> k;
#pragma unroll
    for (int w = 0; w < AS; ++w) {
        k.x[w] = B.x[w * B.cap + i];
        k.z[w] = B.z[w * B.cap + i];
    }
    k.ps = ps_of(B.f[i]);
    return k;
}

template <int AS>
__device__ __forceinline__ bool anticommutes(const u64* x, const u64* z, const GateP<AS>& g) {
    u64 par = 0;
#pragma unroll
    for (int k = 0; k < AS; ++k) par ^= anti_word(x[k], z[k], g.px[k], g.pz[k]);
    return (__popcll(par) & 1) != 0;
}

// Look-back over two 31-bit counters packed as c1 << 31 | c0 (flags in bits
// 62-63).  In/out values use the form c1 << 32 | c0.
__device__ __forceinline__ u64 lookback2(u64* lb, u32 tile, u64 v, int* status) {
    const u64 enc = ((v >> 32) << 31) | (v & 0xffffffffull);
    auto dec = [](u64 e) { return ((e >> 31) & kC31) << 32 | (e & kC31); };
    if (tile == 0) {
        st_volatile64(lb, kF2Pre | enc);
        return 0;
    }
    st_volatile64(lb + tile, kF2Agg | enc);
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
        excl += dec(w & ~(3ull << 62));
        if (fl == 2) break;
        --t;
    }
    const u64 inc = excl + v;
    st_volatile64(lb + tile, kF2Pre | (((inc >> 32) << 31) | (inc & 0xffffffffull)));
    return excl;
}

// ---------------------------------------------------------------------------
// A: expansion into two runs.
// ---------------------------------------------------------------------------
// The look-back of lookback2 run by a whole warp (32 predecessors per round
// trip); every lane returns the exclusive pair of counters.  Bounded.
__device__ __forceinline__ u64 warp_lookback2(u64* lb, u32 tile, u64 v, int* status) {
    const int lane = threadIdx.x & 31;
    const u64 enc = ((v >> 32) << 31) | (v & 0xffffffffull);
    if (tile == 0) {
        if (lane == 0) st_volatile64(lb, kF2Pre | enc);
        return 0;
    }
    if (lane == 0) st_volatile64(lb + tile, kF2Agg | enc);
    u64 excl = 0;
    i64 t = (i64)tile - 1;
    u32 spins = 0;
    while (t >= 0) {
        const i64 q = t - lane;
        const u64 w = q >= 0 ? ld_volatile64(lb + q) : kF2Pre;
        const u32 fl = (u32)(w >> 62);
        const u32 pre = __ballot_sync(0xffffffffu, fl == 2u);
        const u32 zero = __ballot_sync(0xffffffffu, fl == 0u);
        const u32 upto = pre ? (pre & (0u - pre)) * 2u - 1u : 0xffffffffu;
        if (zero & upto) {
            if (++spins > g_spin_limit) {
                if (lane == 0) raise_status(status, PL_ERR_TIMEOUT);
                break;
            }
            if (spins > 64) __nanosleep(64);
            continue;
        }
        u64 c0 = 0, c1 = 0;
        if ((upto >> lane) & 1u) {
            c0 = w & kC31;
            c1 = (w >> 31) & kC31;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            c0 += __shfl_xor_sync(0xffffffffu, c0, o);
            c1 += __shfl_xor_sync(0xffffffffu, c1, o);
        }
        excl += (c1 << 32) | c0;
        if (pre) break;
        t -= 32;
    }
    const u64 inc = excl + v;
    if (lane == 0)
        st_volatile64(lb + tile, kF2Pre | (((inc >> 32) << 31) | (inc & 0xffffffffull)));
    return excl;
}

template <int AS>
__global__ void __launch_bounds__(kPT, AS == 1 ? 4 : 2)
    k_expand(Buf old, const i64* d_m, const GateRec<AS>* table, const int* cursor, Buf r0, Buf r1,
             i64* d_k, u64* lb, u32* ctr, int* status, i64 cap_out, int* d_fail) {
    __shared__ u32 s_tile;
    __shared__ u64 s_warp[kPT / 32];
    __shared__ u64 s_base;
    if (status_set(status)) return;
    const GateRec<AS>& rec = table[*cursor];
    const GateP<AS> g = rec.g;
    const int mode = rec.mode, gate = rec.op;
    const double neg_s = rec.neg_s;
    const bool branching = mode == kGeneral || mode == kHalfPos || mode == kHalfNeg;
    const i64 m = *d_m;
    const u32 ntiles = (u32)((m + kExpTile - 1) / kExpTile);
    if (ntiles == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) d_k[0] = d_k[1] = 0;
        return;
    }
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(ctr, 1u);
        __syncthreads();
        const u32 tile = s_tile;
        __syncthreads();
        if (tile >= ntiles) break;
        const i64 wbase = (i64)tile * kExpTile + warp * (kExpItems * 32);
        u32 amask = 0, cmask = 0, c0 = 0, c1 = 0;
        u32 off0[kExpItems], off1[kExpItems];
#pragma unroll
        for (int t = 0; t < kExpItems; ++t) {
            const i64 j = wbase + t * 32 + lane;
            bool a = false, cl = false;
            if (j < m) {
                u64 x[AS], z[AS];
#pragma unroll
                for (int k = 0; k < AS; ++k) {
                    x[k] = old.x[k * old.cap + j];
                    z[k] = old.z[k * old.cap + j];
                }
                a = branching && anticommutes<AS>(x, z, g);
                const u64 w = g.cls_x ? x[g.cw] : z[g.cw];
                cl = (w & g.cmask) != 0;
            }
            const u32 b0 = __ballot_sync(0xffffffffu, a && !cl);
            const u32 b1 = __ballot_sync(0xffffffffu, a && cl);
            off0[t] = c0 + __popc(b0 & lanemask_lt());
            off1[t] = c1 + __popc(b1 & lanemask_lt());
            c0 += __popc(b0);
            c1 += __popc(b1);
            if (a) amask |= 1u << t;
            if (cl) cmask |= 1u << t;
        }
        if (lane == 0) s_warp[warp] = ((u64)c1 << 32) | c0;
        __syncthreads();
        u64 wpre = 0, tot = 0;
#pragma unroll
        for (int w = 0; w < kPT / 32; ++w) {
            const u64 v = s_warp[w];
            if (w < warp) wpre += v;
            tot += v;
        }
        if (warp == 0) {
            const u64 ex = warp_lookback2(lb, tile, tot, status);
            if (lane == 0) s_base = ex;
        }
        __syncthreads();
        const u64 base = s_base + wpre;
        const i64 base0 = (u32)base, base1 = (u32)(base >> 32);
#pragma unroll
        for (int t = 0; t < kExpItems; ++t) {
            if (!((amask >> t) & 1u)) continue;
            const i64 j = wbase + t * 32 + lane;
            u64 x[AS], z[AS];
#pragma unroll
            for (int k = 0; k < AS; ++k) {
                x[k] = old.x[k * old.cap + j];
                z[k] = old.z[k * old.cap + j];
            }
            const u32 f = old.f[j];
            PhaseAcc acc;
#pragma unroll
            for (int k = 0; k < AS; ++k) acc.step(x[k], z[k], g.px[k], g.pz[k]);
            const u32 fin = mode == kHalfPos ? ((f + 2u) & 3u) : f;
            const u32 nf = acc.phase(fin, g.psf);
            const double nv = mode == kGeneral ? dmul(neg_s, old.v[j]) : old.v[j];
            const bool cl = (cmask >> t) & 1u;
            i64 pos = cl ? base1 + off1[t] : base0 + off0[t];
            // Twin fix-up: the phase-0/phase-1 twins of one string are adjacent
            // in both runs; their children swap order when the phase shift is odd.
            if ((f & 1u) == 0 && j + 1 < m) {
                bool same = true;
#pragma unroll
                for (int k = 0; k < AS; ++k)
                    same = same && old.x[k * old.cap + j + 1] == x[k] &&
                           old.z[k * old.cap + j + 1] == z[k];
                if (same && (nf & 1u)) pos += 1;
            } else if ((f & 1u) == 1 && j > 0) {
                bool same = true;
#pragma unroll
                for (int k = 0; k < AS; ++k)
                    same = same && old.x[k * old.cap + j - 1] == x[k] &&
                           old.z[k * old.cap + j - 1] == z[k];
                if (same && !(nf & 1u)) pos -= 1;
            }
            const Buf& R = cl ? r1 : r0;
            if (pos < 0 || pos >= R.cap) {
                raise_status(status, PL_ERR_INTERNAL);
                continue;
            }
#pragma unroll
            for (int k = 0; k < AS; ++k) {
                R.x[k * R.cap + pos] = x[k] ^ g.px[k];
                R.z[k * R.cap + pos] = z[k] ^ g.pz[k];
            }
            R.f[pos] = (u8)nf;
            R.v[pos] = nv;
        }
        if (tile == ntiles - 1 && tid == 0) {
            const u64 fin = s_base + tot;
            const i64 k0 = (u32)fin, k1 = (u32)(fin >> 32);
            d_k[0] = k0;
            d_k[1] = k1;
            if (m + k0 + k1 > cap_out) {
                raise_status(status, PL_ERR_CAPACITY);
                atomicExch(d_fail, gate);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Merge-path partition: split points of each tile's diagonal range.
// ---------------------------------------------------------------------------
// First i in [lo, hi] with !(A[i] <= B[d-1-i]) (the merge-path split of
// diagonal d, ties taking A first), found by a whole warp: each round tests
// 32 evenly spaced candidates at once, so a split costs about log32(n)
// dependent memory round trips instead of log2(n).  Warp-uniform.
template <int AS>
__device__ __forceinline__ i64 warp_merge_split(const Buf& A, i64 na, const Buf& B, i64 nb,
                                                i64 d) {
    const int lane = threadIdx.x & 31;
    i64 lo = d > nb ? d - nb : 0, hi = d < na ? d : na;
    while (lo < hi) {
        const i64 step = (hi - lo + 31) / 32;
        const i64 i = lo + (i64)lane * step;
        bool p = false;
        if (i < hi) p = kcmp<AS>(gkey<AS>(A, i), gkey<AS>(B, d - 1 - i)) <= 0;
        const int c = __popc(__ballot_sync(0xffffffffu, p));  // the true tests are a prefix
        if (c == 0) break;                                     // pred(lo) is false
        const i64 next = lo + (i64)c * step;
        lo = lo + (i64)(c - 1) * step + 1;
        hi = next < hi ? next : hi;
    }
    return lo;
}

// Splits of the diagonals t*T, t = 0..ntiles (one warp each): tile t merges
// the output range [lo_s[t] + ..., hi_s[t] + ...) of both inputs.
template <int AS>
__global__ void __launch_bounds__(256) k_partition(Buf A, const i64* pa, Buf B, const i64* pb,
                                                   const i64* pb2, int T, u32* lo_s, u32* hi_s,
                                                   u32 max_tiles, const int* status) {
    if (status_set(status)) return;
    const i64 na = *pa, nb = *pb + (pb2 ? *pb2 : 0);
    const i64 total = na + nb;
    const u32 ntiles = (u32)((total + T - 1) / T);
    const int lane = threadIdx.x & 31;
    const u32 nw = (gridDim.x * blockDim.x) >> 5;
    for (u32 t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t <= ntiles; t += nw) {
        const i64 D = (i64)t * T < total ? (i64)t * T : total;
        const u32 sp = (u32)warp_merge_split<AS>(A, na, B, nb, D);
        if (lane == 0) {
            if (t < ntiles && t < max_tiles) lo_s[t] = sp;
            if (t >= 1 && t - 1 < max_tiles) hi_s[t - 1] = sp;
        }
    }
}

// Shared-memory SoA tile of terms.
template <int AS>
struct STile {
    u64* x;  // [AS][cap]
    u64* z;
    double* v;
    u8* f;   // order key bits: bit0 phase, bit1 sign, bit2 removed
    u16* order;
    int cap;
    __device__ __forceinline__ Key<AS> key(int i) const {
        Key<AS> k;
#pragma unroll
        for (int w = 0; w < AS; ++w) {
            k.x[w] = x[w * cap + i];
            k.z[w] = z[w * cap + i];
        }
        k.ps = ps_of(f[i] & 3u);
        return k;
    }
};

template <int AS>
__device__ STile<AS> carve_tile(unsigned char* smem, int cap) {
    STile<AS> S;
    S.cap = cap;
    S.x = reinterpret_cast<u64*>(smem);
    S.z = S.x + AS * cap;
    S.v = reinterpret_cast<double*>(S.z + AS * cap);
    S.f = reinterpret_cast<u8*>(S.v + cap);
    S.order = reinterpret_cast<u16*>(S.f + ((cap + 15) & ~15));
    return S;
}

template <int AS>
constexpr size_t tile_smem_bytes(int cap) {
    return (size_t)cap * (16 * AS + 8) + (size_t)((cap + 15) & ~15) + (size_t)cap * 2 + 64;
}

// Merge [0, na) and [na, na + nb) of the tile into S.order (ties: first part).
template <int AS>
__device__ void block_merge(const STile<AS>& S, int na, int nb) {
    const int L = na + nb;
    const int per = (L + kPT - 1) / kPT;
    const int d = min((int)threadIdx.x * per, L);
    const int e = min(d + per, L);
    int lo = d > nb ? d - nb : 0, hi = d < na ? d : na;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (kcmp<AS>(S.key(mid), S.key(na + d - 1 - mid)) <= 0) lo = mid + 1;
        else hi = mid;
    }
    int a = lo, b = d - lo;
    for (int q = d; q < e; ++q) {
        bool take_a;
        if (a >= na) take_a = false;
        else if (b >= nb) take_a = true;
        else take_a = kcmp<AS>(S.key(a), S.key(na + b)) <= 0;
        S.order[q] = (u16)(take_a ? a++ : na + b++);
    }
}

template <int AS>
__device__ __forceinline__ void tile_load(const STile<AS>& S, int dst, const Buf& B, i64 src) {
#pragma unroll
    for (int w = 0; w < AS; ++w) {
        S.x[w * S.cap + dst] = B.x[w * B.cap + src];
        S.z[w * S.cap + dst] = B.z[w * B.cap + src];
    }
    S.v[dst] = B.v[src];
    S.f[dst] = B.f[src] & 3u;
}

// Stage cnt terms into S: item i < split from A[a_src + i], the rest from
// B[b_src + i - split].  x, z and v by asynchronous copies (all of a
// thread's items in flight at once), the flags byte through registers.
template <int AS, int NL>
__device__ __forceinline__ void tile_load_async(const STile<AS>& S, int cnt, int split,
                                                const Buf& A, i64 a_src, const Buf& B,
                                                i64 b_src) {
    u32 fr[NL];
#pragma unroll
    for (int r = 0; r < NL; ++r) {
        const int i = threadIdx.x + r * kPT;
        fr[r] = 0;
        if (i < cnt) {
            const bool isA = i < split;
            const Buf& G = isA ? A : B;
            const i64 src = isA ? a_src + i : b_src + (i - split);
#pragma unroll
            for (int w = 0; w < AS; ++w) {
                __pipeline_memcpy_async(&S.x[w * S.cap + i], &G.x[w * G.cap + src], 8);
                __pipeline_memcpy_async(&S.z[w * S.cap + i], &G.z[w * G.cap + src], 8);
            }
            __pipeline_memcpy_async(&S.v[i], &G.v[src], 8);
            fr[r] = G.f[src];
        }
    }
    __pipeline_commit();
#pragma unroll
    for (int r = 0; r < NL; ++r) {
        const int i = threadIdx.x + r * kPT;
        if (i < cnt) S.f[i] = (u8)(fr[r] & 3u);
    }
    __pipeline_wait_prior(0);
}

// ---------------------------------------------------------------------------
// B: merge the two runs into one sorted child list.
// ---------------------------------------------------------------------------
template <int AS>
__global__ void __launch_bounds__(kPT, AS == 1 ? 4 : 2)
    k_merge_runs(Buf r0, Buf r1, const i64* d_k, const u32* lo_s, const u32* hi_s, Buf out,
                 u32* ctr, int* status) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ u32 s_tile;
    if (status_set(status)) return;
    constexpr int T = ptile<AS>();
    const STile<AS> S = carve_tile<AS>(smem, T);
    const i64 na = d_k[0], nb = d_k[1], total = na + nb;
    const u32 ntiles = (u32)((total + T - 1) / T);
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(ctr, 1u);
        __syncthreads();
        const u32 tile = s_tile;
        __syncthreads();
        if (tile >= ntiles) break;
        const i64 D = (i64)tile * T;
        const i64 D1 = D + T < total ? D + T : total;
        const i64 a0 = lo_s[tile], a1 = hi_s[tile];
        const i64 b0 = D - a0, b1 = D1 - a1;
        const int la = (int)(a1 - a0), lb = (int)(b1 - b0);
        if (la < 0 || lb < 0 || la + lb > T) {
            raise_status(status, PL_ERR_INTERNAL);
            __syncthreads();
            continue;
        }
        tile_load_async<AS, (T + kPT - 1) / kPT>(S, la + lb, la, r0, a0, r1, b0);
        __syncthreads();
        block_merge<AS>(S, la, lb);
        __syncthreads();
        for (int q = threadIdx.x; q < la + lb; q += kPT) {
            const int e = S.order[q];
            const i64 o = D + q;
            if (o >= out.cap) {
                raise_status(status, PL_ERR_INTERNAL);
                break;
            }
#pragma unroll
            for (int w = 0; w < AS; ++w) {
                out.x[w * out.cap + o] = S.x[w * S.cap + e];
                out.z[w * out.cap + o] = S.z[w * S.cap + e];
            }
            out.f[o] = S.f[e];
            out.v[o] = S.v[e];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// C: merge old terms with the children, reduce, filter, compact.
// ---------------------------------------------------------------------------
__device__ __forceinline__ u32 lookback1(u32* lb, u32 tile, u32 cnt, int* status) {
    constexpr u32 kAgg = 1u << 30, kPre = 2u << 30, kMask = (1u << 30) - 1;
    if (tile == 0) {
        st_volatile(lb, kPre | cnt);
        return 0;
    }
    st_volatile(lb + tile, kAgg | cnt);
    u32 excl = 0;
    i64 t = (i64)tile - 1;
    u32 spins = 0;
    while (t >= 0) {
        const u32 w = ld_volatile(lb + t);
        const u32 fl = w >> 30;
        if (fl == 0) {
            if (++spins > g_spin_limit) {
                raise_status(status, PL_ERR_TIMEOUT);
                break;
            }
            if (spins > 64) __nanosleep(64);
            continue;
        }
        excl += w & kMask;
        if (fl == 2) break;
        --t;
    }
    st_volatile(lb + tile, kPre | ((excl + cnt) & kMask));
    return excl;
}

// Keys of two terms name the same canonical string: (x, z, phase) equal;
// the sign bit of the order key does not take part.
// The same look-back run by a whole warp: each round reads 32 predecessors
// at once, so a tile whose neighbours have only published aggregates still
// finds its prefix in one or two round trips.  All lanes return the
// exclusive prefix.  Bounded.
__device__ __forceinline__ u32 warp_lookback1(u32* lb, u32 tile, u32 cnt, int* status) {
    constexpr u32 kAgg = 1u << 30, kPre = 2u << 30, kMask = (1u << 30) - 1;
    const int lane = threadIdx.x & 31;
    if (tile == 0) {
        if (lane == 0) st_volatile(lb, kPre | cnt);
        return 0;
    }
    if (lane == 0) st_volatile(lb + tile, kAgg | cnt);
    u32 excl = 0;
    i64 t = (i64)tile - 1;  // closest predecessor of this window
    u32 spins = 0;
    while (t >= 0) {
        const i64 q = t - lane;
        const u32 w = q >= 0 ? ld_volatile(lb + q) : kPre;  // before tile 0: prefix 0
        const u32 fl = w >> 30;
        const u32 pre = __ballot_sync(0xffffffffu, fl == 2u);
        const u32 zero = __ballot_sync(0xffffffffu, fl == 0u);
        const u32 upto = pre ? (pre & (0u - pre)) * 2u - 1u : 0xffffffffu;  // lanes <= first prefix
        if (zero & upto) {
            if (++spins > g_spin_limit) {
                if (lane == 0) raise_status(status, PL_ERR_TIMEOUT);
                break;
            }
            if (spins > 64) __nanosleep(64);
            continue;
        }
        u32 v = ((upto >> lane) & 1u) ? (w & kMask) : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        excl += v;
        if (pre) break;
        t -= 32;
    }
    if (lane == 0) st_volatile(lb + tile, kPre | ((excl + cnt) & kMask));
    return excl;
}

template <int AS>
__device__ __forceinline__ bool same_string(const Key<AS>& a, const Key<AS>& b) {
    bool same = ((a.ps ^ b.ps) & 2u) == 0;
#pragma unroll
    for (int w = 0; w < AS; ++w) same = same && a.x[w] == b.x[w] && a.z[w] == b.z[w];
    return same;
}

// Merge of the old terms A (canonical: distinct keys, sign 0) with the sorted
// children C; a string occurs at most once in each, so equal strings meet as
// an adjacent (A, C) pair (ties take A first).  The tile covers merged
// positions [D, D + T); each thread merges IT consecutive positions
// sequentially from shared memory, holding the current A and C keys in
// registers.  A term is a head unless it is a C term whose A predecessor has
// the same string; a head A term adds its C twin (peeked, possibly in the
// next thread's or tile's range).  Each head is reduced as S(sign 0) -
// S(sign 1) of its members in merged order -- the reference's `+=` followed
// by canonicalize -- filtered (zero, cutoff, weight) and compacted with a
// decoupled look-back.
template <int AS>
__global__ void __launch_bounds__(kPT, AS == 1 ? 4 : 2)
    k_merge_reduce(Buf old, const i64* d_m, Buf nw, const i64* d_k, const u32* lo_s,
                   const u32* hi_s, const GateRec<AS>* table, const int* cursor, Buf out,
                   i64* d_out, u64 max_weight, double cutoff, u32* lb, u32* ctr, int* status,
                   int* d_fail) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ u32 s_tile, s_excl;
    __shared__ u32 s_warp[kPT / 32];
    if (status_set(status)) return;
    const GateRec<AS>& rec = table[*cursor];
    const GateP<AS> g = rec.g;
    const int mode = rec.mode, gate = rec.op;
    const double c = rec.c;
    constexpr int IT = PItems<AS>::v;
    constexpr int T = ptile<AS>();
    const STile<AS> S = carve_tile<AS>(smem, T + 2);
    const i64 na = *d_m, nb = d_k[0] + d_k[1], total = na + nb;
    const u32 ntiles = (u32)((total + T - 1) / T);
    if (ntiles == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *d_out = 0;
        return;
    }
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(ctr, 1u);
        __syncthreads();
        const u32 tile = s_tile;
        __syncthreads();
        if (tile >= ntiles) break;
        const i64 D = (i64)tile * T;
        const i64 dend = D + T < total ? D + T : total;
        const i64 a0 = lo_s[tile], a1 = hi_s[tile];
        const i64 b0 = D - a0, b1 = dend - a1;
        const int la = (int)(a1 - a0), lbn = (int)(b1 - b0);
        const int ha = a0 > 0 ? 1 : 0;        // A[a0 - 1] staged before the tile's A terms
        const int hc = b1 < nb ? 1 : 0;       // C[b1] staged after the tile's C terms
        const int cb = ha + la;               // smem index of C[b0]
        const bool bad = la < 0 || lbn < 0 || la + lbn > T || (la + lbn) != (int)(dend - D);
        if (!bad) {
            tile_load_async<AS, (T + 2 + kPT - 1) / kPT>(S, cb + lbn + hc, cb, old, a0 - ha, nw,
                                                         b0);
        }
        __syncthreads();
        // this thread's merged positions [d, d + IT) of the tile
        const int d = tid * IT;
        const int L = bad ? 0 : la + lbn;
        int ai = 0, bi = 0;
        if (d < L) {
            int lo = d > lbn ? d - lbn : 0, hi = d < la ? d : la;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (kcmp<AS>(S.key(ha + mid), S.key(cb + d - 1 - mid)) <= 0) lo = mid + 1;
                else hi = mid;
            }
            ai = lo;
            bi = d - lo;
        }
        Key<AS> ka, kc, kp;  // current A, current C, last A taken (or staged before)
        if (ai < la) ka = S.key(ha + ai);
        if (bi < lbn + hc) kc = S.key(cb + bi);
        bool has_p = ha + ai - 1 >= 0;
        if (has_p) kp = S.key(ha + ai - 1);
        // kept heads: their smem index in S.order[d + j], the reduced value
        // written over the head's own slot (no other thread reads it again)
        u32 nkeep = 0;
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            if (d + it >= L) continue;
            const bool take_a = ai < la && (bi >= lbn || kcmp<AS>(ka, kc) <= 0);
            double sp = 0.0, sm = 0.0;
            bool has = false;
            int e;
            Key<AS> ke;
            if (take_a) {
                e = ha + ai;
                ke = ka;
                // an anticommuting old term is scaled by cos(theta), negated
                // (theta ~ pi) or moved to its child (theta ~ +-pi/2) here,
                // where its merge takes it
                double va = S.v[e];
                bool kept_a = true;
                if (mode != kSkip && anticommutes<AS>(ka.x, ka.z, g)) {
                    if (mode == kGeneral) va = dmul(va, c);
                    else if (mode == kNegate) va = -va;
                    else kept_a = false;
                }
                if (kept_a) {
                    has = true;
                    sp = dadd(sp, va);  // canonical A terms carry sign 0
                }
                // the C twin follows directly (ties take A first)
                if (bi < lbn + hc && same_string<AS>(ka, kc)) {
                    const int ec = cb + bi;
                    const u32 fc = S.f[ec];
                    if (!(fc & 4u)) {
                        has = true;
                        if (fc & 2u) sm = dadd(sm, S.v[ec]);
                        else sp = dadd(sp, S.v[ec]);
                    }
                }
                kp = ka;
                has_p = true;
                ++ai;
                if (ai < la) ka = S.key(ha + ai);
            } else {
                e = cb + bi;
                ke = kc;
                // a C term is a head unless the A term before it is its twin
                const bool twin = has_p && same_string<AS>(kp, kc);
                if (!twin) {
                    const u32 fc = S.f[e];
                    if (!(fc & 4u)) {
                        has = true;
                        if (fc & 2u) sm = dadd(sm, S.v[e]);
                        else sp = dadd(sp, S.v[e]);
                    }
                }
                ++bi;
                if (bi < lbn + hc) kc = S.key(cb + bi);
            }
            if (!has) continue;
            const double rv = dadd(sp, -sm);
            bool k = rv != 0.0;
            if (k && cutoff > 0.0) k = fabs(rv) >= cutoff;
            if (k && max_weight != ~0ull) {
                u64 wsum = 0;
#pragma unroll
                for (int w = 0; w < AS; ++w) wsum += (u64)__popcll(ke.x[w] | ke.z[w]);
                k = wsum <= max_weight;
            }
            if (!k) continue;
            S.order[d + nkeep] = (u16)e;
            S.v[e] = rv;
            ++nkeep;
        }
        // block exclusive scan of per-thread keep counts
        u32 inc = nkeep;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += t;
        }
        if (lane == 31) s_warp[warp] = inc;
        u32 mine[IT];
#pragma unroll
        for (int j = 0; j < IT; ++j) mine[j] = (u32)j < nkeep ? S.order[d + j] : 0u;
        __syncthreads();
        u32 wpre = 0, tot = 0;
#pragma unroll
        for (int w = 0; w < kPT / 32; ++w) {
            const u32 cw = s_warp[w];
            if (w < warp) wpre += cw;
            tot += cw;
        }
        // the tile's kept heads, compacted in output order
        const u32 tbase = wpre + (inc - nkeep);
#pragma unroll
        for (int j = 0; j < IT; ++j)
            if ((u32)j < nkeep) S.order[tbase + j] = (u16)mine[j];
        if (warp == 0) {
            const u32 ex = warp_lookback1(lb, tile, tot, status);
            if (lane == 0) s_excl = ex;
        }
        __syncthreads();
        const i64 obase = (i64)s_excl;
        for (u32 p = tid; p < tot; p += kPT) {
            const int e = S.order[p];
            const i64 o = obase + p;
            if (o >= out.cap) {
                raise_status(status, PL_ERR_CAPACITY);
                atomicExch(d_fail, gate);
                break;
            }
#pragma unroll
            for (int w = 0; w < AS; ++w) {
                out.x[w * out.cap + o] = S.x[w * S.cap + e];
                out.z[w * out.cap + o] = S.z[w * S.cap + e];
            }
            out.f[o] = (u8)(S.f[e] & 1u);
            out.v[o] = S.v[e];
        }
        if (bad && tid == 0) raise_status(status, PL_ERR_INTERNAL);
        if (tile == ntiles - 1 && tid == 0) *d_out = (i64)s_excl + tot;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// In-place and general-path kernels.
// ---------------------------------------------------------------------------
// theta ~ pi: anticommuting terms change sign.  canonical: negate the value
// (canonicalize would fold the sign); otherwise flip the sign bit exactly as
// evolve does (PauliSumOperations.h:124-130).
template <int AS>
__global__ void __launch_bounds__(256) k_negate(Buf b, const i64* d_n, GateP<AS> g, int fold,
                                                const int* status) {
    if (status_set(status)) return;
    const i64 n = *d_n;
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (i64)gridDim.x * blockDim.x) {
        u64 x[AS], z[AS];
#pragma unroll
        for (int k = 0; k < AS; ++k) {
            x[k] = b.x[k * b.cap + i];
            z[k] = b.z[k * b.cap + i];
        }
        if (!anticommutes<AS>(x, z, g)) continue;
        if (fold) b.v[i] = -b.v[i];
        else b.f[i] ^= 2u;
    }
}

// theta ~ +-pi/2 without a following canonicalize: anticommuting Q becomes
// Q*ps in place, with the extra sign flip at +pi/2 (PauliSumOperations.h:131-147).
template <int AS>
__global__ void __launch_bounds__(256) k_halfpi_inplace(Buf b, const i64* d_n, GateP<AS> g,
                                                        int pos, const int* status) {
    if (status_set(status)) return;
    const i64 n = *d_n;
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (i64)gridDim.x * blockDim.x) {
        u64 x[AS], z[AS];
#pragma unroll
        for (int k = 0; k < AS; ++k) {
            x[k] = b.x[k * b.cap + i];
            z[k] = b.z[k * b.cap + i];
        }
        if (!anticommutes<AS>(x, z, g)) continue;
        PhaseAcc acc;
#pragma unroll
        for (int k = 0; k < AS; ++k) {
            acc.step(x[k], z[k], g.px[k], g.pz[k]);
            b.x[k * b.cap + i] = x[k] ^ g.px[k];
            b.z[k * b.cap + i] = z[k] ^ g.pz[k];
        }
        const u32 f = b.f[i];
        b.f[i] = (u8)acc.phase(pos ? (f ^ 2u) : f, g.psf);
    }
}

// General branch materialised: out[0, m) = old terms (anticommuting ones
// scaled by cos), out[m + r] = child r (Q*ps, -sin * value) in old order --
// exactly the array the reference's `+=` sorts (PauliSumCore.h:210-237).
template <int AS>
__global__ void __launch_bounds__(kPT)
    k_materialize(Buf old, i64 m, GateP<AS> g, double c, double neg_s, Buf out, i64* d_total,
                  u64* lb, u32* ctr, int* status) {
    __shared__ u32 s_tile;
    __shared__ u64 s_warp[kPT / 32];
    __shared__ u64 s_base;
    const u32 ntiles = (u32)((m + kExpTile - 1) / kExpTile);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(ctr, 1u);
        __syncthreads();
        const u32 tile = s_tile;
        __syncthreads();
        if (tile >= ntiles) break;
        const i64 wbase = (i64)tile * kExpTile + warp * (kExpItems * 32);
        u32 amask = 0, cnt = 0;
        u32 off[kExpItems];
#pragma unroll
        for (int t = 0; t < kExpItems; ++t) {
            const i64 j = wbase + t * 32 + lane;
            bool a = false;
            if (j < m) {
                u64 x[AS], z[AS];
#pragma unroll
                for (int k = 0; k < AS; ++k) {
                    x[k] = old.x[k * old.cap + j];
                    z[k] = old.z[k * old.cap + j];
                    out.x[k * out.cap + j] = x[k];
                    out.z[k * out.cap + j] = z[k];
                }
                a = anticommutes<AS>(x, z, g);
                out.f[j] = old.f[j];
                out.v[j] = a ? dmul(old.v[j], c) : old.v[j];
            }
            const u32 bal = __ballot_sync(0xffffffffu, a);
            off[t] = cnt + __popc(bal & lanemask_lt());
            cnt += __popc(bal);
            if (a) amask |= 1u << t;
        }
        if (lane == 0) s_warp[warp] = cnt;
        __syncthreads();
        u64 wpre = 0, tot = 0;
#pragma unroll
        for (int w = 0; w < kPT / 32; ++w) {
            const u64 v = s_warp[w];
            if (w < warp) wpre += v;
            tot += v;
        }
        if (tid == 0) s_base = lookback2(lb, tile, tot, status);
        __syncthreads();
        const i64 base = (i64)(u32)(s_base + wpre);
#pragma unroll
        for (int t = 0; t < kExpItems; ++t) {
            if (!((amask >> t) & 1u)) continue;
            const i64 j = wbase + t * 32 + lane;
            const i64 pos = m + base + off[t];
            if (pos >= out.cap) {
                raise_status(status, PL_ERR_CAPACITY);
                continue;
            }
            PhaseAcc acc;
#pragma unroll
            for (int k = 0; k < AS; ++k) {
                const u64 x = old.x[k * old.cap + j], z = old.z[k * old.cap + j];
                acc.step(x, z, g.px[k], g.pz[k]);
                out.x[k * out.cap + pos] = x ^ g.px[k];
                out.z[k * out.cap + pos] = z ^ g.pz[k];
            }
            out.f[pos] = (u8)acc.phase(old.f[j], g.psf);
            out.v[pos] = dmul(neg_s, old.v[j]);
        }
        if (tile == ntiles - 1 && tid == 0) *d_total = m + (i64)(u32)(s_base + tot);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Bulk Clifford gates (PauliSumClifford.h:44-501) as a 16-entry table over
// the Pauli bits (xc, zc, xt, zt) of the gate's qubits: entry e holds the
// new bits (tbits, 4 per entry) and whether the sign flips (tsign bit e).
// The tables are built on the host from each gate's images of X and Z.
// ---------------------------------------------------------------------------
template <int AS>
__global__ void __launch_bounds__(256) k_clifford(Buf b, const i64* d_n, int wc, u64 mc, int wt,
                                                  u64 mt, int two, u64 tbits, u32 tsign,
                                                  const int* status) {
    if (status_set(status)) return;
    const i64 n = *d_n;
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (i64)gridDim.x * blockDim.x) {
        u64 xa = b.x[wc * b.cap + i], za = b.z[wc * b.cap + i];
        u64 xb = xa, zb = za;
        if (two && wt != wc) {
            xb = b.x[wt * b.cap + i];
            zb = b.z[wt * b.cap + i];
        }
        const u32 e = (u32)((xa & mc) != 0) | ((u32)((za & mc) != 0) << 1) |
                      (two ? ((u32)((xb & mt) != 0) << 2) | ((u32)((zb & mt) != 0) << 3) : 0u);
        const u32 o = (u32)(tbits >> (4 * e)) & 15u;
        xa = (xa & ~mc) | ((o & 1u) ? mc : 0ull);
        za = (za & ~mc) | ((o & 2u) ? mc : 0ull);
        if (two) {
            if (wt == wc) {
                xa = (xa & ~mt) | ((o & 4u) ? mt : 0ull);
                za = (za & ~mt) | ((o & 8u) ? mt : 0ull);
            } else {
                b.x[wt * b.cap + i] = (xb & ~mt) | ((o & 4u) ? mt : 0ull);
                b.z[wt * b.cap + i] = (zb & ~mt) | ((o & 8u) ? mt : 0ull);
            }
        }
        b.x[wc * b.cap + i] = xa;
        b.z[wc * b.cap + i] = za;
        b.f[i] ^= (u8)(((tsign >> e) & 1u) << 1);
    }
}

// apply_RX / RY / RZ (PauliSumOperations.h:29-104) materialised:
// out[0, m) = old terms, those anticommuting with P_c scaled by cos(theta/2);
// out[m + r] = the r-th anticommuting term left-multiplied by i P_c
// (multiply_iX / iY / iZ, PauliSumClifford.h:13-40) with sin(theta/2) of its
// original value -- the array the reference's `+=` sorts.  axis 1 X, 2 Y, 3 Z.
template <int AS>
__global__ void __launch_bounds__(kPT)
    k_materialize_rgate(Buf old, i64 m, int w, u64 mk, int axis, double ch, double sh, Buf out,
                        i64* d_total, u64* lb, u32* ctr, int* status) {
    __shared__ u32 s_tile;
    __shared__ u64 s_warp[kPT / 32];
    __shared__ u64 s_base;
    const u32 ntiles = (u32)((m + kExpTile - 1) / kExpTile);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(ctr, 1u);
        __syncthreads();
        const u32 tile = s_tile;
        __syncthreads();
        if (tile >= ntiles) break;
        const i64 wbase = (i64)tile * kExpTile + warp * (kExpItems * 32);
        u32 amask = 0, cnt = 0;
        u32 off[kExpItems];
#pragma unroll
        for (int t = 0; t < kExpItems; ++t) {
            const i64 j = wbase + t * 32 + lane;
            bool a = false;
            if (j < m) {
#pragma unroll
                for (int k = 0; k < AS; ++k) {
                    out.x[k * out.cap + j] = old.x[k * old.cap + j];
                    out.z[k * out.cap + j] = old.z[k * old.cap + j];
                }
                const bool xc = (old.x[w * old.cap + j] & mk) != 0;
                const bool zc = (old.z[w * old.cap + j] & mk) != 0;
                a = axis == 3 ? xc : (axis == 1 ? zc : (xc != zc));
                out.f[j] = old.f[j];
                out.v[j] = a ? dmul(old.v[j], ch) : old.v[j];
            }
            const u32 bal = __ballot_sync(0xffffffffu, a);
            off[t] = cnt + __popc(bal & lanemask_lt());
            cnt += __popc(bal);
            if (a) amask |= 1u << t;
        }
        if (lane == 0) s_warp[warp] = cnt;
        __syncthreads();
        u64 wpre = 0, tot = 0;
#pragma unroll
        for (int q = 0; q < kPT / 32; ++q) {
            const u64 v = s_warp[q];
            if (q < warp) wpre += v;
            tot += v;
        }
        if (warp == 0) {
            const u64 ex = warp_lookback2(lb, tile, tot, status);
            if (lane == 0) s_base = ex;
        }
        __syncthreads();
        const i64 base = (i64)(u32)(s_base + wpre);
#pragma unroll
        for (int t = 0; t < kExpItems; ++t) {
            if (!((amask >> t) & 1u)) continue;
            const i64 j = wbase + t * 32 + lane;
            const i64 pos = m + base + off[t];
            if (pos >= out.cap) {
                raise_status(status, PL_ERR_CAPACITY);
                continue;
            }
#pragma unroll
            for (int k = 0; k < AS; ++k) {
                out.x[k * out.cap + pos] = old.x[k * old.cap + j];
                out.z[k * out.cap + pos] = old.z[k * old.cap + j];
            }
            const bool xc = (old.x[w * old.cap + j] & mk) != 0;
            const bool zc = (old.z[w * old.cap + j] & mk) != 0;
            u32 f = old.f[j];
            if (axis == 3) {
                f ^= (u32)(!zc) << 1;
                out.z[w * out.cap + pos] ^= mk;
            } else if (axis == 1) {
                f ^= (u32)xc << 1;
                out.x[w * out.cap + pos] ^= mk;
            } else {
                f ^= (u32)(!xc) << 1;
                out.x[w * out.cap + pos] ^= mk;
                out.z[w * out.cap + pos] ^= mk;
            }
            out.f[pos] = (u8)f;
            out.v[pos] = dmul(old.v[j], sh);
        }
        if (tile == ntiles - 1 && tid == 0) *d_total = m + (i64)(u32)(s_base + tot);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Reductions over a sum's terms: basis_state_expectation, trace, lookup and
// frobenius_norm2 (PauliSumUtils.h:178-268, 400-410), and the join of
// trace_product (PauliSumUtils.h:412-447).  Each thread sums its strided
// terms in order, blocks reduce with a fixed tree and one block adds the
// block sums in order: a deterministic order (not the reference's term
// order, so results agree within rounding).
// ---------------------------------------------------------------------------
enum RedKind : int {
    kRedBasis = 0,
    kRedTrace = 1,
    kRedFrob = 2,
    kRedLookup = 3,
    kRedCountAbove = 4,  // terms with |c| >= threshold (exact below 2^53)
    kRedMaxAbs = 5       // largest |c| (combined with max, not +)
};
constexpr int kRedBlocks = 296;

struct RedArgs {
    int kind;
    u32 qf;             // lookup: flags of the query
    u64 bits[kMaxAS];   // basis state, one bit per qubit
    u64 qx[kMaxAS];     // lookup: the query string
    u64 qz[kMaxAS];
    double threshold;   // count above
};

template <int AS>
__device__ __forceinline__ double red_term(const Buf& b, i64 i, const RedArgs& R) {
    const u32 f = b.f[i];
    const double v = b.v[i];
    if (R.kind == kRedFrob) return dmul(v, v);
    if (R.kind == kRedCountAbove) return fabs(v) >= R.threshold ? 1.0 : 0.0;
    if (R.kind == kRedMaxAbs) return fabs(v);
    if (R.kind == kRedLookup) {
        bool match = true;
#pragma unroll
        for (int k = 0; k < AS; ++k)
            match = match && b.x[k * b.cap + i] == R.qx[k] && b.z[k * b.cap + i] == R.qz[k];
        if (!match) return 0.0;
        const u32 rel = (f - R.qf) & 3u;
        if (rel & 1u) return 0.0;
        return (rel & 2u) ? -v : v;
    }
    // basis state / trace: real-phase terms without X (and, for trace, without Z)
    u64 xs = 0, zs = 0;
    u32 par = 0;
#pragma unroll
    for (int k = 0; k < AS; ++k) {
        const u64 z = b.z[k * b.cap + i];
        xs |= b.x[k * b.cap + i];
        zs |= z;
        par ^= (u32)__popcll(z & R.bits[k]);
    }
    if (xs != 0 || (f & 1u)) return 0.0;
    if (R.kind == kRedTrace && zs != 0) return 0.0;
    const bool neg = ((f >> 1) & 1u) ^ (R.kind == kRedBasis ? (par & 1u) : 0u);
    return neg ? -v : v;
}

__device__ __forceinline__ double red_op(double a, double b, bool use_max) {
    return use_max ? fmax(a, b) : dadd(a, b);
}

__device__ __forceinline__ double block_tree_sum(double a, double* sm, bool use_max = false) {
    sm[threadIdx.x] = a;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st)
            sm[threadIdx.x] = red_op(sm[threadIdx.x], sm[threadIdx.x + st], use_max);
        __syncthreads();
    }
    return sm[0];
}

template <int AS>
__global__ void __launch_bounds__(256) k_reduce_terms(Buf b, const i64* d_n, RedArgs R,
                                                      double* partial) {
    __shared__ double sm[256];
    const i64 n = *d_n;
    const bool mx = R.kind == kRedMaxAbs;
    double acc = 0.0;
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (i64)gridDim.x * blockDim.x)
        acc = red_op(acc, red_term<AS>(b, i, R), mx);
    const double s = block_tree_sum(acc, sm, mx);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// The block sums in order, times 2^exp2.
__global__ void __launch_bounds__(256) k_sum_partials(const double* partial, int np, int exp2,
                                                      double* out, int use_max) {
    __shared__ double sm[256];
    double acc = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) acc = red_op(acc, partial[i], use_max);
    const double s = block_tree_sum(acc, sm, use_max != 0);
    if (threadIdx.x == 0) *out = scalbn(s, exp2);
}

// trace_product join: A canonical (sorted by (x, z, phase), sign folded into
// the value), so the complex weight of a pattern is (value of its phase-0
// entry, value of its phase-1 entry).  Each term of B finds its pattern by
// binary search and adds Re(w * c_b * i^k_b).
template <int AS>
__device__ __forceinline__ int xz_cmp(const Buf& a, i64 i, const u64* x, const u64* z) {
#pragma unroll
    for (int k = 0; k < AS; ++k) {
        const u64 v = a.x[k * a.cap + i];
        if (v != x[k]) return v < x[k] ? -1 : 1;
    }
#pragma unroll
    for (int k = 0; k < AS; ++k) {
        const u64 v = a.z[k * a.cap + i];
        if (v != z[k]) return v < z[k] ? -1 : 1;
    }
    return 0;
}

template <int AS>
__global__ void __launch_bounds__(256) k_trace_join(Buf A, const i64* d_na, Buf B,
                                                    const i64* d_nb, double* partial) {
    __shared__ double sm[256];
    const i64 na = *d_na, nb = *d_nb;
    double acc = 0.0;
    for (i64 j = (i64)blockIdx.x * blockDim.x + threadIdx.x; j < nb;
         j += (i64)gridDim.x * blockDim.x) {
        u64 x[AS], z[AS];
#pragma unroll
        for (int k = 0; k < AS; ++k) {
            x[k] = B.x[k * B.cap + j];
            z[k] = B.z[k * B.cap + j];
        }
        i64 lo = 0, hi = na;  // first entry of A with (x, z) >= the pattern
        while (lo < hi) {
            const i64 mid = (lo + hi) >> 1;
            if (xz_cmp<AS>(A, mid, x, z) < 0) lo = mid + 1;
            else hi = mid;
        }
        double re = 0.0, im = 0.0;
        for (i64 i = lo; i < na && i < lo + 2 && xz_cmp<AS>(A, i, x, z) == 0; ++i) {
            if (A.f[i] & 1u) im = A.v[i];
            else re = A.v[i];
        }
        const double v = B.v[j];
        double c;
        switch (B.f[j] & 3u) {
            case 0: c = dmul(re, v); break;
            case 1: c = -dmul(im, v); break;
            case 2: c = -dmul(re, v); break;
            default: c = dmul(im, v); break;
        }
        acc = dadd(acc, c);
    }
    const double s = block_tree_sum(acc, sm);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// Order-preserving filters cutoff / truncate_weight (PauliSumUtils.h:378-393).
template <int AS>
__global__ void __launch_bounds__(kPT) k_filter(Buf in, i64 n, Buf out, double eps,
                                                u64 max_weight, i64* d_out, u32* lb, u32* ctr,
                                                int* status) {
    __shared__ u32 s_tile, s_excl;
    __shared__ u32 s_warp[kPT / 32];
    const u32 ntiles = (u32)((n + kExpTile - 1) / kExpTile);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(ctr, 1u);
        __syncthreads();
        const u32 tile = s_tile;
        __syncthreads();
        if (tile >= ntiles) break;
        const i64 wbase = (i64)tile * kExpTile + warp * (kExpItems * 32);
        u32 kmask = 0, cnt = 0;
        u32 off[kExpItems];
#pragma unroll
        for (int t = 0; t < kExpItems; ++t) {
            const i64 j = wbase + t * 32 + lane;
            bool k = false;
            if (j < n) {
                k = true;
                if (eps > 0.0) k = fabs(in.v[j]) >= eps;
                if (k && max_weight != ~0ull) {
                    u64 w = 0;
#pragma unroll
                    for (int q = 0; q < AS; ++q)
                        w += (u64)__popcll(in.x[q * in.cap + j] | in.z[q * in.cap + j]);
                    k = w <= max_weight;
                }
            }
            const u32 bal = __ballot_sync(0xffffffffu, k);
            off[t] = cnt + __popc(bal & lanemask_lt());
            cnt += __popc(bal);
            if (k) kmask |= 1u << t;
        }
        if (lane == 0) s_warp[warp] = cnt;
        __syncthreads();
        u32 wpre = 0, tot = 0;
#pragma unroll
        for (int w = 0; w < kPT / 32; ++w) {
            const u32 v = s_warp[w];
            if (w < warp) wpre += v;
            tot += v;
        }
        if (tid == 0) s_excl = lookback1(lb, tile, tot, status);
        __syncthreads();
#pragma unroll
        for (int t = 0; t < kExpItems; ++t) {
            if (!((kmask >> t) & 1u)) continue;
            const i64 j = wbase + t * 32 + lane;
            const i64 o = (i64)s_excl + wpre + off[t];
#pragma unroll
            for (int q = 0; q < AS; ++q) {
                out.x[q * out.cap + o] = in.x[q * in.cap + j];
                out.z[q * out.cap + o] = in.z[q * in.cap + j];
            }
            out.f[o] = in.f[j];
            out.v[o] = in.v[j];
        }
        if (tile == ntiles - 1 && tid == 0) *d_out = (i64)s_excl + tot;
        __syncthreads();
    }
}

template <int AS>
__global__ void __launch_bounds__(256) k_cnot_state(Buf b, const i64* d_n, int wc, u64 mc,
                                                    int wt, u64 mt, const int* status) {
    if (status_set(status)) return;
    const i64 n = *d_n;
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (i64)gridDim.x * blockDim.x) {
        const u64 xc = (b.x[wc * b.cap + i] & mc) != 0, zc = (b.z[wc * b.cap + i] & mc) != 0;
        const u64 xt = (b.x[wt * b.cap + i] & mt) != 0, zt = (b.z[wt * b.cap + i] & mt) != 0;
        b.f[i] ^= (u8)((xc & zt & (1ull ^ xt ^ zc)) << 1);
        b.x[wt * b.cap + i] ^= (0ull - xc) & mt;
        b.z[wc * b.cap + i] ^= (0ull - zt) & mc;
    }
}

// Start of a fast-path rotation: zero the look-back words and tile counters
// of the chain and select its gate record (idx >= 0: op idx; idx < 0: the
// op after the current one, which is how a captured chain advances).
__global__ void __launch_bounds__(256) k_rot_begin(uint4* zero, size_t n16, int* cursor,
                                                   int idx) {
    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16;
         i += (size_t)gridDim.x * blockDim.x)
        zero[i] = z;
    if (blockIdx.x == 0 && threadIdx.x == 0) *cursor = idx >= 0 ? idx : *cursor + 1;
}

__global__ void k_set_int(int* p, int v) { *p = v; }

// The sizes of the rotation the cursor names: terms in, anticommuting terms
// (children), terms out after the merge and truncation.
__global__ void k_log_gate(i64* log, i64 nlog, const int* cursor, const i64* n_in,
                           const i64* k, const i64* n_out) {
    const int q = *cursor;
    if (q < 0 || q >= nlog) return;
    log[3 * q] = *n_in;
    log[3 * q + 1] = k[0] + k[1];
    log[3 * q + 2] = *n_out;
}

// A layer of CNOTs (PauliSumClifford.h:213-239) applied in op order to each
// term in one pass: pairs[2k] = control, pairs[2k+1] = target.
template <int AS>
__global__ void __launch_bounds__(256) k_cnot_layer(Buf b, const i64* d_n, const int* pairs,
                                                    int count, const int* status) {
    if (status_set(status)) return;
    const i64 n = *d_n;
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (i64)gridDim.x * blockDim.x) {
        u64 x[AS], z[AS];
#pragma unroll
        for (int k = 0; k < AS; ++k) {
            x[k] = b.x[k * b.cap + i];
            z[k] = b.z[k * b.cap + i];
        }
        u32 f = b.f[i];
        for (int q = 0; q < count; ++q) {
            const int c = pairs[2 * q], t = pairs[2 * q + 1];
            const int wc = c >> 6, wt = t >> 6;
            const u64 mc = 1ull << (c & 63), mt = 1ull << (t & 63);
            u64 xwc = 0, zwc = 0, xwt = 0, zwt = 0;
#pragma unroll
            for (int k = 0; k < AS; ++k) {
                if (k == wc) { xwc = x[k]; zwc = z[k]; }
                if (k == wt) { xwt = x[k]; zwt = z[k]; }
            }
            const u64 xc = (xwc & mc) != 0, zc = (zwc & mc) != 0;
            const u64 xt = (xwt & mt) != 0, zt = (zwt & mt) != 0;
            f ^= (u32)((xc & zt & (1ull ^ xt ^ zc)) << 1);
#pragma unroll
            for (int k = 0; k < AS; ++k) {
                if (k == wt) x[k] ^= (0ull - xc) & mt;
                if (k == wc) z[k] ^= (0ull - zt) & mc;
            }
        }
#pragma unroll
        for (int k = 0; k < AS; ++k) {
            b.x[k * b.cap + i] = x[k];
            b.z[k * b.cap + i] = z[k];
        }
        b.f[i] = (u8)f;
    }
}

// ---------------------------------------------------------------------------
// trim(max_terms[, keep]) (PauliSumUtils.h:331-375): keep the max_terms terms
// of largest |c| in their original order.  The reference's nth_element leaves
// the choice among equal |c| at the boundary to the library; here (as in the
// oracle) ties go to the lower index.  Terms whose (x, z) is in the protect
// list are always kept and do not count against the rest's budget.
//
// The magnitude's bit pattern (sign cleared) orders like |c|, so the
// threshold is a radix select over 64-bit keys: kTrimPasses histogram passes
// of up to 11 bits, each followed by a one-block pick of the bin holding the
// k-th largest.  Then per-tile counts of keys above / equal to the threshold,
// one scan, and an order-preserving emit.  Every step reads the term count
// from the device, so no host round trip is needed.
// ---------------------------------------------------------------------------
constexpr int kTrimBits = 11;
constexpr int kTrimBins = 1 << kTrimBits;
constexpr int kTrimPasses = (64 + kTrimBits - 1) / kTrimBits;  // 6
constexpr int kTrimItems = 8;
constexpr u32 kTrimTile = kPT * kTrimItems;

struct TrimCtl {
    u64 prefix;     // key bits decided so far
    u64 k;          // how many still to select below the decided prefix
    u64 T;          // threshold key (after the last pick)
    u64 r;          // how many keys == T are kept
    u64 protected_n;
    int keep_all;   // n - protected <= budget: every term survives
    int pad;
    u32 hist[kTrimBins];
};

struct Protect {
    const u64* x;  // sorted (x words, z words) of the protected strings
    const u64* z;
    i64 n;         // 0: nothing protected
    i64 stride;
};

__device__ __forceinline__ u64 mag_key(double v) {
    return (u64)__double_as_longlong(v) & 0x7fffffffffffffffull;
}

template <int AS>
__device__ __forceinline__ bool is_protected(const Protect& P, const u64* x, const u64* z) {
    i64 lo = 0, hi = P.n;
    while (lo < hi) {
        const i64 mid = (lo + hi) >> 1;
        int c = 0;
#pragma unroll
        for (int w = 0; w < AS; ++w) {
            const u64 a = P.x[w * P.stride + mid];
            if (c == 0 && a != x[w]) c = a < x[w] ? -1 : 1;
        }
#pragma unroll
        for (int w = 0; w < AS; ++w) {
            const u64 a = P.z[w * P.stride + mid];
            if (c == 0 && a != z[w]) c = a < z[w] ? -1 : 1;
        }
        if (c == 0) return true;
        if (c < 0) lo = mid + 1;
        else hi = mid;
    }
    return false;
}

template <int AS>
__device__ __forceinline__ bool term_protected(const Buf& b, i64 i, const Protect& P) {
    if (P.n == 0) return false;
    u64 x[AS], z[AS];
#pragma unroll
    for (int w = 0; w < AS; ++w) {
        x[w] = b.x[w * b.cap + i];
        z[w] = b.z[w * b.cap + i];
    }
    return is_protected<AS>(P, x, z);
}

// Count the protected terms and set up the select.
template <int AS>
__global__ void __launch_bounds__(256) k_trim_init(Buf b, const i64* d_n, u64 max_terms,
                                                   Protect P, TrimCtl* C, const int* status) {
    if (status_set(status)) return;
    const i64 n = *d_n;
    u32 cnt = 0;
    if (P.n > 0)
        for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
             i += (i64)gridDim.x * blockDim.x)
            cnt += term_protected<AS>(b, i, P) ? 1u : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd((unsigned long long*)&C->protected_n, cnt);
}

__global__ void __launch_bounds__(256) k_trim_setup(const i64* d_n, u64 max_terms, TrimCtl* C) {
    const i64 n = *d_n;
    const u64 prot = C->protected_n;
    const u64 rest = (u64)n - prot;
    const u64 budget = max_terms > prot ? max_terms - prot : 0;
    for (int i = threadIdx.x; i < kTrimBins; i += blockDim.x) C->hist[i] = 0;
    if (threadIdx.x == 0) {
        C->prefix = 0;
        C->k = budget;
        C->keep_all = (u64)n <= max_terms || rest <= budget;
        C->T = 0;
        C->r = 0;
    }
}

// Histogram of key bits [shift, shift + bits) over unprotected keys whose
// bits above shift + bits equal the decided prefix.
template <int AS>
__global__ void __launch_bounds__(256) k_trim_hist(Buf b, const i64* d_n, Protect P, TrimCtl* C,
                                                   int shift, int bits) {
    __shared__ u32 sh[kTrimBins];
    if (C->keep_all || C->k == 0) return;
    for (int i = threadIdx.x; i < kTrimBins; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const i64 n = *d_n;
    const int hi = shift + bits;
    const u64 pre = C->prefix;
    const u32 dmask = (1u << bits) - 1u;
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (i64)gridDim.x * blockDim.x) {
        const u64 key = mag_key(b.v[i]);
        if (hi < 64 && (key >> hi) != (pre >> hi)) continue;
        if (term_protected<AS>(b, i, P)) continue;
        atomicAdd(&sh[(u32)(key >> shift) & dmask], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kTrimBins; i += blockDim.x)
        if (sh[i]) atomicAdd(&C->hist[i], sh[i]);
}

// One block: the bin (from the top) holding the k-th largest key.
__global__ void __launch_bounds__(32) k_trim_pick(TrimCtl* C, int shift, int bits, int last) {
    if (C->keep_all) return;
    if (threadIdx.x == 0) {
        u64 k = C->k;
        if (k > 0) {
            const int nb = 1 << bits;
            u64 cum = 0;
            int bin = 0;
            for (int d = nb - 1; d >= 0; --d) {
                const u64 c = C->hist[d];
                if (cum + c >= k) {
                    bin = d;
                    break;
                }
                cum += c;
            }
            C->prefix |= (u64)bin << shift;
            C->k = k - cum;
        }
        if (last) {
            // k == 0 (nothing to select): no unprotected key survives
            C->T = C->k == 0 ? ~0ull : C->prefix;
            C->r = C->k;
        }
    }
    __syncwarp();
    for (int i = threadIdx.x; i < kTrimBins; i += 32) C->hist[i] = 0;
}

__device__ __forceinline__ bool trim_above(const TrimCtl& C, u64 key) {
    return C.keep_all || (C.T != ~0ull && key > C.T);
}
__device__ __forceinline__ bool trim_tie(const TrimCtl& C, u64 key) {
    return !C.keep_all && C.T != ~0ull && key == C.T;
}

// Per tile: terms kept for sure (above the threshold or protected) and ties.
template <int AS>
__global__ void __launch_bounds__(kPT) k_trim_count(Buf b, const i64* d_n, Protect P,
                                                    const TrimCtl* Cp, u32* gt, u32* eq,
                                                    const int* status) {
    __shared__ u32 s_gt[kPT / 32], s_eq[kPT / 32];
    if (status_set(status)) return;
    const TrimCtl& C = *Cp;
    const i64 n = *d_n;
    const u32 ntiles = (u32)((n + kTrimTile - 1) / kTrimTile);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (u32 tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const i64 wbase = (i64)tile * kTrimTile + warp * (kTrimItems * 32);
        u32 g = 0, e = 0;
#pragma unroll
        for (int t = 0; t < kTrimItems; ++t) {
            const i64 i = wbase + t * 32 + lane;
            if (i >= n) continue;
            const u64 key = mag_key(b.v[i]);
            if (trim_above(C, key) || term_protected<AS>(b, i, P)) ++g;
            else if (trim_tie(C, key)) ++e;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            g += __shfl_xor_sync(0xffffffffu, g, o);
            e += __shfl_xor_sync(0xffffffffu, e, o);
        }
        if (lane == 0) {
            s_gt[warp] = g;
            s_eq[warp] = e;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            u32 tg = 0, te = 0;
            for (int w = 0; w < kPT / 32; ++w) {
                tg += s_gt[w];
                te += s_eq[w];
            }
            gt[tile] = tg;
            eq[tile] = te;
        }
        __syncthreads();
    }
}

// One block: tie offsets, kept counts and kept offsets per tile; the output
// size.  eq[] is replaced by its exclusive scan, gt[] by the kept offsets.
__global__ void __launch_bounds__(1024) k_trim_scan(const i64* d_n, const TrimCtl* Cp, u32* gt,
                                                    u32* eq, i64* d_out, const int* status) {
    __shared__ u32 sw[33];
    __shared__ u64 s_carry[2];
    if (status_set(status)) return;
    const i64 n = *d_n;
    const u32 ntiles = (u32)((n + kTrimTile - 1) / kTrimTile);
    const u64 r = Cp->r;
    if (threadIdx.x == 0) s_carry[0] = s_carry[1] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (u32 base = 0; base < ntiles; base += 1024) {
        const u32 t = base + threadIdx.x;
        const u32 e = t < ntiles ? eq[t] : 0u;
        const u32 g = t < ntiles ? gt[t] : 0u;
        // scan of ties
        u32 inc = e;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 v = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += v;
        }
        if (lane == 31) sw[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            u32 c = sw[lane], ci = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const u32 v = __shfl_up_sync(0xffffffffu, ci, o);
                if (lane >= o) ci += v;
            }
            sw[lane] = ci - c;
            if (lane == 31) sw[32] = ci;
        }
        __syncthreads();
        const u64 eoff = s_carry[0] + sw[warp] + (inc - e);
        const u32 etot = sw[32];
        __syncthreads();
        const u64 keep_ties = eoff >= r ? 0 : (r - eoff < e ? r - eoff : e);
        const u32 kept = g + (u32)keep_ties;
        // scan of kept
        inc = kept;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 v = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += v;
        }
        if (lane == 31) sw[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            u32 c = sw[lane], ci = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const u32 v = __shfl_up_sync(0xffffffffu, ci, o);
                if (lane >= o) ci += v;
            }
            sw[lane] = ci - c;
            if (lane == 31) sw[32] = ci;
        }
        __syncthreads();
        const u64 koff = s_carry[1] + sw[warp] + (inc - kept);
        const u32 ktot = sw[32];
        if (t < ntiles) {
            eq[t] = (u32)eoff;
            gt[t] = (u32)koff;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_carry[0] += etot;
            s_carry[1] += ktot;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *d_out = (i64)s_carry[1];
}

// Order-preserving emit of the survivors into out.
template <int AS>
__global__ void __launch_bounds__(kPT) k_trim_emit(Buf b, const i64* d_n, Protect P,
                                                   const TrimCtl* Cp, const u32* koff,
                                                   const u32* eoff, Buf out, int* status) {
    __shared__ u32 s_k[kPT / 32], s_e[kPT / 32];
    if (status_set(status)) return;
    const TrimCtl& C = *Cp;
    const i64 n = *d_n;
    const u32 ntiles = (u32)((n + kTrimTile - 1) / kTrimTile);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (u32 tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const i64 wbase = (i64)tile * kTrimTile + warp * (kTrimItems * 32);
        // warp prefix of ties and of sure survivors, in item order
        u32 sure = 0, tie = 0;
        u32 cs = 0, ce = 0;
#pragma unroll
        for (int t = 0; t < kTrimItems; ++t) {
            const i64 i = wbase + t * 32 + lane;
            bool s = false, e = false;
            if (i < n) {
                const u64 key = mag_key(b.v[i]);
                s = trim_above(C, key) || term_protected<AS>(b, i, P);
                e = !s && trim_tie(C, key);
            }
            const u32 bs = __ballot_sync(0xffffffffu, s), be = __ballot_sync(0xffffffffu, e);
            if (s) sure |= 1u << t;
            if (e) tie |= 1u << t;
            cs += __popc(bs);
            ce += __popc(be);
        }
        if (lane == 0) {
            s_k[warp] = cs;
            s_e[warp] = ce;
        }
        __syncthreads();
        u32 we = 0;
        for (int w = 0; w < warp; ++w) we += s_e[w];
        // ties before this warp, then kept terms before this warp
        const u64 tie0 = (u64)eoff[tile] + we;
        u32 wk = 0;
        {
            // kept before this warp = sure before + ties kept before
            u32 ties_before = 0, sure_before = 0;
            for (int w = 0; w < warp; ++w) {
                sure_before += s_k[w];
                ties_before += s_e[w];
            }
            const u64 e0 = (u64)eoff[tile];
            const u64 kt = e0 >= C.r ? 0 : (C.r - e0 < ties_before ? C.r - e0 : ties_before);
            wk = sure_before + (u32)kt;
        }
        u64 o = (u64)koff[tile] + wk;
        u64 tr = tie0;  // rank of the next tie
#pragma unroll
        for (int t = 0; t < kTrimItems; ++t) {
            const i64 i = wbase + t * 32 + lane;
            const bool s = (sure >> t) & 1u, e = (tie >> t) & 1u;
            const u32 be = __ballot_sync(0xffffffffu, e);
            const u64 my_rank = tr + __popc(be & lanemask_lt());
            const bool keep = s || (e && my_rank < C.r);
            const u32 bk = __ballot_sync(0xffffffffu, keep);
            const u64 pos = o + __popc(bk & lanemask_lt());
            if (keep) {
                if ((i64)pos >= out.cap) {
                    raise_status(status, PL_ERR_INTERNAL);
                } else {
#pragma unroll
                    for (int w = 0; w < AS; ++w) {
                        out.x[w * out.cap + pos] = b.x[w * b.cap + i];
                        out.z[w * out.cap + pos] = b.z[w * b.cap + i];
                    }
                    out.f[pos] = b.f[i];
                    out.v[pos] = b.v[i];
                }
            }
            o += __popc(bk);
            tr += __popc(be);
        }
        __syncthreads();
    }
}

// ---- Clifford gate tables ------------------------------------------------
// A Clifford gate maps each generator X_c, Z_c, X_t, Z_t to a signed Pauli
// (its image); conjugation is multiplicative, so the image of any Pauli is
// the product of its generators' images.  Paulis are kept in product form
// i^k X_c^x0 Z_c^z0 X_t^x1 Z_t^z1; a term's bits (Y = (1,1)) read as
// i^{#Y} X^x Z^z since Y = i X Z.
struct P2 {
    unsigned x[2], z[2], k;
};

P2 p2_mul(const P2& a, const P2& b) {
    P2 r;
    r.k = (a.k + b.k) & 3u;
    for (int q = 0; q < 2; ++q) {
        r.k = (r.k + 2u * (a.z[q] & b.x[q])) & 3u;  // Z X = -X Z
        r.x[q] = a.x[q] ^ b.x[q];
        r.z[q] = a.z[q] ^ b.z[q];
    }
    return r;
}

// Signed string "[-]PQ" (P on c, Q on t) in product form.
P2 p2_of(const char* s) {
    P2 r{{0, 0}, {0, 0}, 0};
    unsigned sign = 0;
    if (*s == '-') {
        sign = 1;
        ++s;
    }
    unsigned ny = 0;
    for (int q = 0; q < 2 && s[q]; ++q) {
        r.x[q] = s[q] == 'X' || s[q] == 'Y';
        r.z[q] = s[q] == 'Z' || s[q] == 'Y';
        ny += s[q] == 'Y';
    }
    r.k = (ny + 2u * sign) & 3u;
    return r;
}

struct GateImages {
    const char* img[4];  // images of X_c, Z_c, X_t, Z_t
};

// Generator images of PL_GATE_1 .. PL_GATE_SWAP, read off the reference's
// gate definitions (PauliSumClifford.h:44-490) and its truth-table tests.
const GateImages kGateImages[] = {
    {{"XI", "ZI", "IX", "IZ"}},      // unused (0)
    {{"ZI", "XI", "IX", "IZ"}},      // H
    {{"YI", "ZI", "IX", "IZ"}},      // S
    {{"-XI", "YI", "IX", "IZ"}},     // H_YZ
    {{"YI", "-ZI", "IX", "IZ"}},     // H_XY
    {{"XI", "-YI", "IX", "IZ"}},     // sqrt(X)
    {{"-ZI", "XI", "IX", "IZ"}},     // sqrt(Y)
    {{"XI", "-ZI", "IX", "IZ"}},     // X
    {{"-XI", "-ZI", "IX", "IZ"}},    // Y
    {{"-XI", "ZI", "IX", "IZ"}},     // Z
    {{"XI", "ZI", "IX", "IZ"}},      // I
    {{"XX", "ZI", "IX", "ZZ"}},      // CNOT
    {{"XZ", "ZI", "ZX", "IZ"}},      // CZ
    {{"XY", "ZI", "ZX", "ZZ"}},      // CY
    {{"XI", "ZX", "IX", "XZ"}},      // XC_X
    {{"XI", "ZY", "XX", "XZ"}},      // XC_Y
    {{"XI", "ZZ", "XX", "IZ"}},      // XC_Z
    {{"XX", "ZX", "IX", "YZ"}},      // YC_X
    {{"XY", "ZY", "YX", "YZ"}},      // YC_Y
    {{"XZ", "ZZ", "YX", "IZ"}},      // YC_Z
    {{"IX", "IZ", "XI", "ZI"}},      // SWAP
};

// Image of the term bits e = xc | zc << 1 | xt << 2 | zt << 3 under gate g:
// new bits and sign flip.
void gate_apply(int g, unsigned e, unsigned* out_bits, unsigned* sign) {
    const GateImages& G = kGateImages[g];
    const unsigned b[4] = {e & 1u, (e >> 1) & 1u, (e >> 2) & 1u, (e >> 3) & 1u};
    P2 r{{0, 0}, {0, 0}, (b[0] & b[1]) + (b[2] & b[3])};  // i^{#Y}
    for (int k = 0; k < 4; ++k)
        if (b[k]) r = p2_mul(r, p2_of(G.img[k]));
    const unsigned ny = (r.x[0] & r.z[0]) + (r.x[1] & r.z[1]);
    *out_bits = r.x[0] | (r.z[0] << 1) | (r.x[1] << 2) | (r.z[1] << 3);
    *sign = ((r.k + 4u - ny) & 3u) >> 1;  // a Clifford image of a Hermitian Pauli: 0 or 2
}

// Packed table of gate g (iSWAP = SWAP, CZ, S on c, S on t;
// PauliSumClifford.h:493-499).
void gate_table(int g, u64* tbits, u32* tsign) {
    *tbits = 0;
    *tsign = 0;
    for (unsigned e = 0; e < 16; ++e) {
        unsigned bits = e, sg = 0;
        if (g == PL_GATE_ISWAP) {
            unsigned s1;
            gate_apply(PL_GATE_SWAP, bits, &bits, &s1);
            sg ^= s1;
            gate_apply(PL_GATE_CZ, bits, &bits, &s1);
            sg ^= s1;
            gate_apply(PL_GATE_S, bits, &bits, &s1);
            sg ^= s1;
            unsigned hi = bits >> 2, nb;
            gate_apply(PL_GATE_S, hi, &nb, &s1);
            bits = (bits & 3u) | ((nb & 3u) << 2);
            sg ^= s1;
        } else {
            gate_apply(g, bits, &bits, &sg);
        }
        *tbits |= (u64)bits << (4 * e);
        *tsign |= (sg & 1u) << e;
    }
}

// isCloseOne (PauliSumOperations.h:19-21).
bool close_one(double v) { return std::fabs(v - 1.0) <= 1e-14; }

}  // namespace
}  // namespace pl

// ===========================================================================
// Host state
// ===========================================================================
using namespace pl;

struct pl_state {
    int as = 1;
    cudaStream_t st = nullptr;
    i64 cap = 0;
    void* mem = nullptr;
    Buf S[2], R0, R1, N;
    int cur = 0;
    i64* d_size = nullptr;  // [2]: sizes of S[0], S[1]
    i64* d_k = nullptr;     // [2]: run sizes
    i64* d_tmp = nullptr;   // scratch count
    int* d_status = nullptr;
    int* d_fail = nullptr;
    u64* lbA = nullptr;
    u32* lbC = nullptr;
    u32* ctr = nullptr;     // [8]
    u32 *spB_lo = nullptr, *spB_hi = nullptr, *spC_lo = nullptr, *spC_hi = nullptr;
    u32 max_tiles = 0;
    size_t zero_bytes = 0;  // bytes from lbA to the end of the counters (one memset per gate)
    DevArena ws;            // collate workspace
    // 0: anything; 1: distinct (x,z,phase) keys; 2: canonical and sorted
    int cls = 0;
    int* d_cursor = nullptr;  // op whose gate record the fast-path kernels read
    void* d_table = nullptr;  // gate records of the running propagation (one per op)
    size_t table_bytes = 0;
    int* d_pairs = nullptr;   // CNOT (control, target) per op
    size_t pairs_bytes = 0;
    bool use_graphs = false;
    // Captured rotation chains keyed by (length, start buffer, max_weight,
    // cutoff bits); they hold the buffer pointers, so growing drops them.
    std::map<std::tuple<int, int, uint64_t, uint64_t>, cudaGraphExec_t> graphs;
    pl::MemBudget* budget = nullptr;
    size_t held_bytes = 0;    // device bytes of mem (counted against budget)
    cudaStream_t cap_st = nullptr;  // private stream the chains are captured on
    void* trim_mem = nullptr;       // trim control block and per-tile counts
    size_t trim_bytes = 0;
    double* red = nullptr;          // block sums and the result of a reduction
    // Per-op sizes of the fast-path rotations (PL_OPT_GATE_LOG): terms in,
    // anticommuting terms, terms out, three i64 per op in processing order.
    bool gate_log = false;
    i64* d_log = nullptr;
    i64 log_ops = 0;       // ops the log holds
    i64 log_used = 0;      // ops of the last propagation
    const volatile int32_t* cancel = nullptr;  // pl_state_set_cancel_flag
    // Terms at the last host read of the size: the chain kernels' grids are
    // sized from it (their tile loops cover any size, so a stale value only
    // costs speed, never correctness).
    i64 size_hint = 0;
};

namespace pl {
namespace {

inline size_t a256(size_t b) { return (b + 255) & ~size_t(255); }

size_t buf_bytes(int as, i64 cap) {
    return 2 * a256(8 * (size_t)as * cap) + a256(cap) + a256(8 * (size_t)cap);
}

Buf carve_buf(unsigned char*& p, int as, i64 cap) {
    Buf b;
    b.cap = cap;
    b.x = (u64*)p;
    p += a256(8 * (size_t)as * cap);
    b.z = (u64*)p;
    p += a256(8 * (size_t)as * cap);
    b.v = (double*)p;
    p += a256(8 * (size_t)cap);
    b.f = (u8*)p;
    p += a256(cap);
    return b;
}

// Allocate all buffers for capacity cap (contents undefined).
size_t state_bytes(int as, i64 cap) {
    const u32 max_tiles = (u32)((2 * cap) / 256 + 4);
    const size_t small = a256(8 * (size_t)max_tiles) + a256(4 * (size_t)max_tiles) +
                         a256(4 * 16) + 4 * a256(4 * (size_t)max_tiles) + a256(8 * 8) + a256(64);
    return 5 * buf_bytes(as, cap) + small;
}

int state_alloc(pl_state* s, i64 cap, void** mem_out, Buf* S, Buf& R0, Buf& R1, Buf& N,
                size_t* small_off) {
    const size_t total = state_bytes(s->as, cap);
    void* mem = nullptr;
    if (dev_alloc(&mem, total, s->st) != cudaSuccess) {
        cudaGetLastError();
        return record_status(PL_ERR_OOM, "pl_state buffers");
    }
    unsigned char* p = (unsigned char*)mem;
    S[0] = carve_buf(p, s->as, cap);
    S[1] = carve_buf(p, s->as, cap);
    R0 = carve_buf(p, s->as, cap);
    R1 = carve_buf(p, s->as, cap);
    N = carve_buf(p, s->as, cap);
    *small_off = (size_t)(p - (unsigned char*)mem);
    *mem_out = mem;
    return PL_OK;
}

void wire_small(pl_state* s, unsigned char* p, u32 max_tiles) {
    s->max_tiles = max_tiles;
    unsigned char* z0 = p;
    s->lbA = (u64*)p;
    p += a256(8 * (size_t)max_tiles);
    s->lbC = (u32*)p;
    p += a256(4 * (size_t)max_tiles);
    s->ctr = (u32*)p;
    p += a256(4 * 16);
    s->zero_bytes = (size_t)(p - z0);
    s->spB_lo = (u32*)p;
    p += a256(4 * (size_t)max_tiles);
    s->spB_hi = (u32*)p;
    p += a256(4 * (size_t)max_tiles);
    s->spC_lo = (u32*)p;
    p += a256(4 * (size_t)max_tiles);
    s->spC_hi = (u32*)p;
    p += a256(4 * (size_t)max_tiles);
    s->d_size = (i64*)p;
    s->d_k = s->d_size + 2;
    s->d_tmp = s->d_size + 4;
    p += a256(8 * 8);
    s->d_status = (int*)p;
    s->d_fail = s->d_status + 1;
    s->d_cursor = s->d_status + 2;
}

void drop_graphs(pl_state* s) {
    for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second);
    s->graphs.clear();
}

// (Re)build all buffers with capacity >= need, keeping the current state.
int state_grow(pl_state* s, i64 need) {
    i64 cap = std::max<i64>(need, std::max<i64>(2 * s->cap, 1 << 16));
    i64 n = 0;
    if (s->mem) {
        PL_CUDA_TRY(cudaMemcpyAsync(&n, s->d_size + s->cur, sizeof(i64), cudaMemcpyDeviceToHost,
                                    s->st));
        PL_CUDA_TRY(cudaStreamSynchronize(s->st));
    }
    void* mem = nullptr;
    Buf S[2], R0, R1, N;
    size_t off = 0;
    const size_t nbytes = state_bytes(s->as, cap);
    if (s->budget) s->budget->resize(s->held_bytes, nbytes);
    const int rc = state_alloc(s, cap, &mem, S, R0, R1, N, &off);
    if (rc) {
        if (s->budget) s->budget->resize(nbytes, s->held_bytes);
        return rc;
    }
    drop_graphs(s);
    int status = 0, fail = 0;
    if (s->mem) {
        const Buf& o = s->S[s->cur];
        if (n > 0) {
            PL_CUDA_TRY(cudaMemcpy2DAsync(S[0].x, 8 * cap, o.x, 8 * o.cap, 8 * n, s->as,
                                          cudaMemcpyDeviceToDevice, s->st));
            PL_CUDA_TRY(cudaMemcpy2DAsync(S[0].z, 8 * cap, o.z, 8 * o.cap, 8 * n, s->as,
                                          cudaMemcpyDeviceToDevice, s->st));
            PL_CUDA_TRY(cudaMemcpyAsync(S[0].f, o.f, n, cudaMemcpyDeviceToDevice, s->st));
            PL_CUDA_TRY(cudaMemcpyAsync(S[0].v, o.v, 8 * n, cudaMemcpyDeviceToDevice, s->st));
        }
        PL_CUDA_TRY(cudaMemcpyAsync(&status, s->d_status, sizeof(int), cudaMemcpyDeviceToHost,
                                    s->st));
        PL_CUDA_TRY(cudaStreamSynchronize(s->st));
        dev_free(s->mem, s->st);
    }
    s->mem = mem;
    s->held_bytes = nbytes;
    s->cap = cap;
    s->S[0] = S[0];
    s->S[1] = S[1];
    s->R0 = R0;
    s->R1 = R1;
    s->N = N;
    s->cur = 0;
    wire_small(s, (unsigned char*)mem + off, (u32)((2 * cap) / 256 + 4));
    i64 sizes[8] = {n, 0, 0, 0, 0, 0, 0, 0};
    int st2[2] = {status == PL_ERR_CAPACITY ? 0 : status, fail};
    PL_CUDA_TRY(cudaMemcpyAsync(s->d_size, sizes, sizeof(sizes), cudaMemcpyHostToDevice, s->st));
    PL_CUDA_TRY(cudaMemcpyAsync(s->d_status, st2, sizeof(st2), cudaMemcpyHostToDevice, s->st));
    PL_CUDA_TRY(cudaStreamSynchronize(s->st));
    return PL_OK;
}

int read_size(pl_state* s, i64* n) {
    PL_CUDA_TRY(cudaMemcpyAsync(n, s->d_size + s->cur, sizeof(i64), cudaMemcpyDeviceToHost, s->st));
    PL_CUDA_TRY(cudaStreamSynchronize(s->st));
    s->size_hint = *n;
    return PL_OK;
}

// Status word, failing op and the current size in one synchronisation.
int read_status_size(pl_state* s, int* status, int* fail) {
    int v[2] = {0, 0};
    i64 n = 0;
    PL_CUDA_TRY(cudaMemcpyAsync(v, s->d_status, sizeof(v), cudaMemcpyDeviceToHost, s->st));
    PL_CUDA_TRY(cudaMemcpyAsync(&n, s->d_size + s->cur, sizeof(i64), cudaMemcpyDeviceToHost,
                                s->st));
    PL_CUDA_TRY(cudaStreamSynchronize(s->st));
    *status = v[0];
    *fail = v[1];
    if (v[0] == 0) s->size_hint = n;
    return PL_OK;
}

int read_status(pl_state* s, int* status, int* fail) {
    int v[2] = {0, 0};
    PL_CUDA_TRY(cudaMemcpyAsync(v, s->d_status, sizeof(v), cudaMemcpyDeviceToHost, s->st));
    PL_CUDA_TRY(cudaStreamSynchronize(s->st));
    *status = v[0];
    *fail = v[1];
    return PL_OK;
}

int clear_status(pl_state* s) {
    PL_CUDA_TRY(cudaMemsetAsync(s->d_status, 0, 2 * sizeof(int), s->st));
    return PL_OK;
}

SoAView view_of(const Buf& b, i64 n) { return SoAView{b.x, b.z, b.f, b.v, n, b.cap}; }
SoAOut out_of(const Buf& b) { return SoAOut{b.x, b.z, b.f, b.v, b.cap}; }

// Collate S[cur] (n terms, host-known) into S[other].
int state_collate(pl_state* s, i64 n, const CollateArgs& a) {
    if (n > s->cap) return record_status(PL_ERR_INTERNAL, "state_collate size");
    const size_t need = collate_ws_bytes(s->as, n);
    const size_t ws_before = s->ws.bytes;
    if (need > ws_before && s->budget) s->budget->resize(s->held_bytes + ws_before, s->held_bytes + need);
    int rc = s->ws.ensure(need);
    if (rc) {
        if (need > ws_before && s->budget) s->budget->resize(s->held_bytes + need, s->held_bytes + ws_before);
        return rc;
    }
    const int other = 1 - s->cur;
    i64 cnt = 0;
    cudaEvent_t e0 = timed_begin(s->st);
    rc = collate_soa(s->as, view_of(s->S[s->cur], n), out_of(s->S[other]), a, &cnt, s->ws.ptr,
                     s->ws.bytes, s->st);
    if (rc) return rc;
    timed_end(e0, s->st, "state_collate_span", 0ull);
    PL_CUDA_TRY(cudaMemcpyAsync(s->d_size + other, &cnt, sizeof(i64), cudaMemcpyHostToDevice,
                                s->st));
    PL_CUDA_TRY(cudaStreamSynchronize(s->st));
    s->cur = other;
    return PL_OK;
}

struct Rot {
    std::vector<u64> px, pz;
    u32 pf;
    double theta;
};

template <int AS>
GateP<AS> make_gate(const Rot& r, bool* single) {
    GateP<AS> g;
    int bits = 0, cw = 0;
    u64 cm = 0;
    int cls_x = 1;
    for (int k = 0; k < AS; ++k) {
        g.px[k] = r.px[k];
        g.pz[k] = r.pz[k];
    }
    // the class bit: the generator's first set x bit, else its first z bit
    for (int k = 0; k < AS && !cm; ++k)
        if (r.px[k]) {
            cw = k;
            cm = r.px[k] & (~r.px[k] + 1);
            cls_x = 1;
        }
    for (int k = 0; k < AS && !cm; ++k)
        if (r.pz[k]) {
            cw = k;
            cm = r.pz[k] & (~r.pz[k] + 1);
            cls_x = 0;
        }
    for (int k = 0; k < AS; ++k) bits += __builtin_popcountll(r.px[k] | r.pz[k]);
    g.psf = (r.pf ^ 1u) & 3u;
    g.cw = cw;
    g.cmask = cm;
    g.cls_x = cls_x;
    *single = bits == 1;
    return g;
}

int classify(double theta, double* c, double* sn) {
    *c = std::cos(theta);
    *sn = std::sin(theta);
    if (close_one(*c)) return kSkip;
    if (close_one(-*c)) return kNegate;
    if (close_one(*sn)) return kHalfPos;
    if (close_one(-*sn)) return kHalfNeg;
    return kGeneral;
}

int grid_persistent(int per_sm) { return sm_count() * per_sm; }

template <int AS>
int set_smem_attrs() {
    static thread_local bool done[kMaxAS + 1] = {};
    if (done[AS]) return PL_OK;
    constexpr int T = ptile<AS>();
    PL_CUDA_TRY(cudaFuncSetAttribute(k_merge_runs<AS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)tile_smem_bytes<AS>(T)));
    PL_CUDA_TRY(cudaFuncSetAttribute(k_merge_reduce<AS>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)tile_smem_bytes<AS>(T + 2)));
    PL_CUDA_TRY(cudaFuncSetAttribute(k_merge_reduce<AS>,
                                     cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    PL_CUDA_TRY(cudaFuncSetAttribute(k_merge_runs<AS>,
                                     cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    done[AS] = true;
    return PL_OK;
}

// One fast-path rotation on a canonical state, S[in] -> S[1-in], reading its
// gate record table[op] (op < 0: the record after the current one).  With
// timed = false nothing but kernels is issued, so the chain can be captured.
template <int AS>
int rotation_chain(pl_state* s, int in, int op, const pl_truncation& tr, bool timed) {
    const int outb = 1 - in;
    constexpr int T = ptile<AS>();
    const auto* table = static_cast<const GateRec<AS>*>(s->d_table);
    int pgrid = std::max(1, std::min((int)((s->max_tiles + 8) / 8), sm_count() * 8));
    const int full = grid_persistent(AS == 1 ? 4 : 2);
    int gexp = full, gruns = full, gred = full;
    if (timed) {
        // launched kernel by kernel: grids for the terms the chain can meet
        // before the next size read (a small state leaves the SMs to other
        // lanes' kernels); a captured chain keeps full grids, as it is
        // replayed at every size
        const i64 est = 4 * s->size_hint + 65536;
        auto cl = [](i64 v, int hi) { return (int)std::max<i64>(1, std::min<i64>(v, hi)); };
        gexp = cl((est + kExpTile - 1) / kExpTile, full);
        gruns = cl((est + T - 1) / T, full);
        gred = cl((2 * est + T - 1) / T, full);
        pgrid = cl((2 * est / T + 8) / 8 + 1, pgrid);
    }
    const u64 mw = tr.max_weight;
    const double cut = tr.coefficient_cutoff > 0.0 ? tr.coefficient_cutoff : 0.0;
    cudaEvent_t e0 = timed ? timed_begin(s->st) : nullptr;
    k_rot_begin<<<sm_count(), 256, 0, s->st>>>(reinterpret_cast<uint4*>(s->lbA), s->zero_bytes / 16,
                                               s->d_cursor, op);
    k_expand<AS><<<gexp, kPT, 0, s->st>>>(
        s->S[in], s->d_size + in, table, s->d_cursor, s->R0, s->R1, s->d_k, s->lbA, s->ctr + 0,
        s->d_status, s->cap, s->d_fail);
    if (timed) timed_end(e0, s->st, "k_expand", 0ull);
    e0 = timed ? timed_begin(s->st) : nullptr;
    k_partition<AS><<<pgrid, 256, 0, s->st>>>(s->R0, s->d_k, s->R1, s->d_k + 1, nullptr, T,
                                              s->spB_lo, s->spB_hi, s->max_tiles, s->d_status);
    k_merge_runs<AS><<<gruns, kPT, tile_smem_bytes<AS>(T), s->st>>>(
        s->R0, s->R1, s->d_k, s->spB_lo, s->spB_hi, s->N, s->ctr + 1, s->d_status);
    k_partition<AS><<<pgrid, 256, 0, s->st>>>(s->S[in], s->d_size + in, s->N, s->d_k, s->d_k + 1,
                                              T, s->spC_lo, s->spC_hi, s->max_tiles, s->d_status);
    if (timed) timed_end(e0, s->st, "k_merge_runs+partitions", 0ull);
    e0 = timed ? timed_begin(s->st) : nullptr;
    k_merge_reduce<AS><<<gred, kPT, tile_smem_bytes<AS>(T + 2), s->st>>>(
        s->S[in], s->d_size + in, s->N, s->d_k, s->spC_lo, s->spC_hi, table, s->d_cursor,
        s->S[outb], s->d_size + outb, mw, cut, s->lbC, s->ctr + 2, s->d_status, s->d_fail);
    if (timed) timed_end(e0, s->st, "k_merge_reduce", 0ull);
    pl::note_launches(6);
    if (s->gate_log && s->d_log) {
        k_log_gate<<<1, 1, 0, s->st>>>(s->d_log, s->log_ops, s->d_cursor, s->d_size + in,
                                        s->d_k, s->d_size + outb);
        pl::note_launch();
    }
    return PL_OK;
}
constexpr int kChainKernels = 6;

// A run of len fast-path rotations starting at op first.  Whole chunks of
// kGraphChunk rotations replay one captured CUDA graph (captured once per
// start buffer and truncation for the state's current buffers; an even
// chunk ends on the buffer it started from, so the same graph serves every
// chunk of every run); the graphs advance the device cursor themselves.
// The rest of the run is launched kernel by kernel.
constexpr int kGraphChunk = 8;

template <int AS>
int rotation_graph(pl_state* s, int first, int len, const pl_truncation& tr) {
    const double cut = tr.coefficient_cutoff > 0.0 ? tr.coefficient_cutoff : 0.0;
    u64 cut_bits;
    std::memcpy(&cut_bits, &cut, sizeof(cut_bits));
    const int chunks = len / kGraphChunk;
    if (chunks > 0) {
        const auto key =
            std::make_tuple(kGraphChunk, s->cur, (uint64_t)tr.max_weight, (uint64_t)cut_bits);
        auto it = s->graphs.find(key);
        cudaGraphExec_t ex = nullptr;
        if (it != s->graphs.end()) {
            ex = it->second;
        } else {
            // Capture on a private stream (the caller's may be the legacy
            // default stream, which cannot be captured); the graph then runs
            // on s->st.
            if (!s->cap_st)
                PL_CUDA_TRY(cudaStreamCreateWithFlags(&s->cap_st, cudaStreamNonBlocking));
            capture_lock();
            const cudaError_t eb =
                cudaStreamBeginCapture(s->cap_st, cudaStreamCaptureModeThreadLocal);
            if (eb != cudaSuccess) {
                capture_unlock();
                return record_cuda(eb);
            }
            const cudaStream_t user_st = s->st;
            s->st = s->cap_st;
            int in = s->cur;
            for (int r = 0; r < kGraphChunk; ++r) {
                rotation_chain<AS>(s, in, -1, tr, false);
                in = 1 - in;
            }
            s->st = user_st;
            cudaGraph_t g = nullptr;
            const cudaError_t ec = cudaStreamEndCapture(s->cap_st, &g);
            capture_unlock();
            if (ec != cudaSuccess) return record_cuda(ec);
            const cudaError_t ei = cudaGraphInstantiate(&ex, g, 0);
            cudaGraphDestroy(g);
            if (ei != cudaSuccess) return record_cuda(ei);
            s->graphs[key] = ex;
        }
        k_set_int<<<1, 1, 0, s->st>>>(s->d_cursor, first - 1);
        pl::note_launch();
        for (int c = 0; c < chunks; ++c) PL_CUDA_TRY(cudaGraphLaunch(ex, s->st));
        pl::note_launches((unsigned long long)(kChainKernels + (s->gate_log ? 1 : 0)) *
                          kGraphChunk * chunks);
    }
    for (int r = chunks * kGraphChunk; r < len; ++r) {
        const int rc = rotation_chain<AS>(s, s->cur, first + r, tr, true);
        if (rc) return rc;
        s->cur ^= 1;
    }
    return PL_OK;
}

// General-path rotation (any state, any generator) with or without the
// following apply_truncation.
template <int AS>
int general_rotation(pl_state* s, const Rot& r, bool truncate, const pl_truncation& tr,
                     i64* k_anti = nullptr) {
    bool single = false;
    const GateP<AS> g = make_gate<AS>(r, &single);
    double c, sn;
    const int mode = classify(r.theta, &c, &sn);
    i64 n = 0;
    int rc = read_size(s, &n);
    if (rc) return rc;
    const int grid = grid_for(n, 256, sm_count() * 8);
    if (mode == kNegate) {
        k_negate<AS><<<grid, 256, 0, s->st>>>(s->S[s->cur], s->d_size + s->cur, g, 0,
                                              s->d_status), pl::note_launch();
        if (s->cls == 2) s->cls = 1;
    } else if (mode == kHalfPos || mode == kHalfNeg) {
        k_halfpi_inplace<AS><<<grid, 256, 0, s->st>>>(s->S[s->cur], s->d_size + s->cur, g,
                                                      mode == kHalfPos, s->d_status), pl::note_launch();
        if (s->cls == 2) s->cls = 1;
    } else if (mode == kGeneral) {
        // old + children can need up to 2n slots
        if (2 * n > s->cap) {
            rc = state_grow(s, 2 * n);
            if (rc) return rc;
        }
        PL_CUDA_TRY(cudaMemsetAsync(s->lbA, 0, s->zero_bytes, s->st));
        const int other = 1 - s->cur;
        k_materialize<AS><<<grid_persistent(4), kPT, 0, s->st>>>(
            s->S[s->cur], n, g, c, -sn, s->S[other], s->d_tmp, s->lbA, s->ctr + 0, s->d_status), pl::note_launch();
        i64 total = 0;
        PL_CUDA_TRY(cudaMemcpyAsync(&total, s->d_tmp, sizeof(i64), cudaMemcpyDeviceToHost, s->st));
        int st[2];
        PL_CUDA_TRY(cudaMemcpyAsync(st, s->d_status, sizeof(st), cudaMemcpyDeviceToHost, s->st));
        PL_CUDA_TRY(cudaStreamSynchronize(s->st));
        if (n == 0) total = 0;
        if (st[0]) return record_status(st[0], "evolve: materialise");
        if (k_anti) *k_anti = total - n;
        s->cur = other;
        CollateArgs a;
        if (truncate) {
            a.mode = kProp;
            a.cutoff = tr.coefficient_cutoff > 0.0 ? tr.coefficient_cutoff : 0.0;
            a.max_weight = tr.max_weight;
        } else {
            a.mode = kCombine;
        }
        rc = state_collate(s, total, a);
        if (rc) return rc;
        s->cls = truncate ? 2 : 0;
        return PL_OK;
    }
    PL_CUDA_TRY(cudaGetLastError());
    if (!truncate) return PL_OK;
    // apply_truncation after a fast-path branch
    rc = read_size(s, &n);
    if (rc) return rc;
    CollateArgs a;
    a.mode = kCanon;
    a.cutoff = tr.coefficient_cutoff > 0.0 ? tr.coefficient_cutoff : 0.0;
    a.max_weight = tr.max_weight;
    rc = state_collate(s, n, a);
    if (rc) return rc;
    s->cls = 2;
    return PL_OK;
}

// trim(max_terms[, protect]) of S[cur] into S[1-cur], all on the stream (the
// term count stays on the device).  Terms kept in their original order.
template <int AS>
int trim_state(pl_state* s, u64 max_terms, const Protect& P) {
    const size_t tiles = (size_t)(s->cap / kTrimTile) + 2;
    const size_t need = a256(sizeof(TrimCtl)) + 2 * a256(4 * tiles);
    if (need > s->trim_bytes) {
        if (s->trim_mem) dev_free(s->trim_mem, s->st);
        s->trim_mem = nullptr;
        s->trim_bytes = 0;
        PL_CUDA_TRY(dev_alloc(&s->trim_mem, need, s->st));
        s->trim_bytes = need;
    }
    auto* C = static_cast<TrimCtl*>(s->trim_mem);
    u32* gt = reinterpret_cast<u32*>(static_cast<unsigned char*>(s->trim_mem) +
                                     a256(sizeof(TrimCtl)));
    u32* eq = gt + a256(4 * tiles) / 4;
    const int in = s->cur, outb = 1 - s->cur;
    const i64* d_n = s->d_size + in;
    PL_CUDA_TRY(cudaMemsetAsync(C, 0, offsetof(TrimCtl, hist), s->st));
    if (P.n > 0)
        k_trim_init<AS><<<grid_persistent(4), 256, 0, s->st>>>(s->S[in], d_n, max_terms, P, C,
                                                               s->d_status), pl::note_launch();
    k_trim_setup<<<1, 256, 0, s->st>>>(d_n, max_terms, C), pl::note_launch();
    for (int p = 0; p < kTrimPasses; ++p) {
        const int shift = std::max(0, 64 - kTrimBits * (p + 1));
        const int bits = 64 - kTrimBits * p - shift;
        k_trim_hist<AS><<<grid_persistent(4), 256, 0, s->st>>>(s->S[in], d_n, P, C, shift, bits),
            pl::note_launch();
        k_trim_pick<<<1, 32, 0, s->st>>>(C, shift, bits, p == kTrimPasses - 1), pl::note_launch();
    }
    k_trim_count<AS><<<grid_persistent(4), kPT, 0, s->st>>>(s->S[in], d_n, P, C, gt, eq,
                                                           s->d_status), pl::note_launch();
    k_trim_scan<<<1, 1024, 0, s->st>>>(d_n, C, gt, eq, s->d_size + outb, s->d_status),
        pl::note_launch();
    k_trim_emit<AS><<<grid_persistent(4), kPT, 0, s->st>>>(s->S[in], d_n, P, C, gt, eq,
                                                          s->S[outb], s->d_status),
        pl::note_launch();
    PL_CUDA_TRY(cudaGetLastError());
    s->cur = outb;
    return PL_OK;
}

// Make a state of class 1 (distinct keys) canonical: sort by (x, z, phase),
// folding signs (values then carry the sign; see the header comment).
int state_canonical_sort(pl_state* s) {
    i64 n = 0;
    int rc = read_size(s, &n);
    if (rc) return rc;
    CollateArgs a;
    a.mode = kCanon;
    rc = state_collate(s, n, a);
    if (rc) return rc;
    s->cls = 2;
    return PL_OK;
}

struct Op {
    int kind;  // 0 rotation, 1 CNOT, 2 Clifford gate `gate`
    int a, b;
    int gate;
};

// Device copies of the op tables (gate records, CNOT pairs), grow-only with
// headroom; captured graphs hold the table pointer, so a reallocation drops
// them.
template <int AS>
int upload_tables(pl_state* s, const std::vector<GateRec<AS>>& recs,
                  const std::vector<int>& pairs) {
    const size_t tb = sizeof(GateRec<AS>) * std::max<size_t>(recs.size(), 1);
    const size_t pb = sizeof(int) * std::max<size_t>(pairs.size(), 2);
    if (tb > s->table_bytes || pb > s->pairs_bytes) {
        PL_CUDA_TRY(cudaStreamSynchronize(s->st));
        drop_graphs(s);
        if (s->d_table) dev_free(s->d_table, s->st);
        if (s->d_pairs) dev_free(s->d_pairs, s->st);
        s->d_table = nullptr;
        s->d_pairs = nullptr;
        s->table_bytes = s->pairs_bytes = 0;
        const size_t tcap = std::max(tb, sizeof(GateRec<AS>) * 16384);
        const size_t pcap = std::max(pb, sizeof(int) * 2 * 16384);
        PL_CUDA_TRY(dev_alloc(&s->d_table, tcap, s->st));
        PL_CUDA_TRY(dev_alloc(reinterpret_cast<void**>(&s->d_pairs), pcap, s->st));
        s->table_bytes = tcap;
        s->pairs_bytes = pcap;
    }
    // pageable sources: the calls return once the data is staged
    PL_CUDA_TRY(cudaMemcpyAsync(s->d_table, recs.data(), sizeof(GateRec<AS>) * recs.size(),
                                cudaMemcpyHostToDevice, s->st));
    PL_CUDA_TRY(cudaMemcpyAsync(s->d_pairs, pairs.data(), sizeof(int) * pairs.size(),
                                cudaMemcpyHostToDevice, s->st));
    return PL_OK;
}

constexpr int kGraphMin = 8;  // shortest run of rotations replayed from a graph

template <int AS>
int run_ops(pl_state* s, const std::vector<Rot>& rots, const std::vector<Op>& ops,
            const pl_truncation& tr) {
    const bool trimming = tr.max_terms != ~0ull;
    const Protect no_protect{nullptr, nullptr, 0, 0};
    int rc = set_smem_attrs<AS>();
    if (rc) return rc;
    // per-rotation parameters, then one record per op for the device
    std::vector<GateP<AS>> gates(rots.size());
    std::vector<int> modes(rots.size()), singles(rots.size());
    std::vector<double> cs(rots.size()), sns(rots.size());
    for (size_t r = 0; r < rots.size(); ++r) {
        bool single = false;
        gates[r] = make_gate<AS>(rots[r], &single);
        singles[r] = single;
        modes[r] = classify(rots[r].theta, &cs[r], &sns[r]);
    }
    if (ops.empty()) return PL_OK;
    {
        i64 n0 = 0;  // the size the first chains' grids are sized from
        rc = read_size(s, &n0);
        if (rc) return rc;
    }
    if (s->gate_log) {
        if (s->log_ops < (i64)ops.size()) {
            // captured chains hold the log's address
            drop_graphs(s);
            if (s->d_log) dev_free(s->d_log, s->st);
            s->d_log = nullptr;
            s->log_ops = 0;
            void* p = nullptr;
            if (dev_alloc(&p, 24 * ops.size(), s->st) != cudaSuccess) {
                cudaGetLastError();
                return record_status(PL_ERR_OOM, "propagate: gate log");
            }
            s->d_log = static_cast<i64*>(p);
            s->log_ops = (i64)ops.size();
        }
        PL_CUDA_TRY(fill32_async(s->d_log, 0u, 24 * ops.size(), s->st));
        s->log_used = (i64)ops.size();
    }
    {
        std::vector<GateRec<AS>> recs(ops.size());
        std::vector<int> pairs(2 * ops.size(), 0);
        for (size_t q = 0; q < ops.size(); ++q) {
            std::memset(&recs[q], 0, sizeof(recs[q]));
            if (ops[q].kind == 1) {
                pairs[2 * q] = ops[q].a;
                pairs[2 * q + 1] = ops[q].b;
            } else if (ops[q].kind == 0) {
                const int r = ops[q].a;
                recs[q].g = gates[r];
                recs[q].mode = modes[r];
                recs[q].op = (int)q;
                recs[q].c = cs[r];
                recs[q].neg_s = -sns[r];
            }
        }
        rc = upload_tables<AS>(s, recs, pairs);
        if (rc) return rc;
    }
    constexpr int kWindow = 192;
    std::vector<int> in_buf(ops.size(), 0);
    size_t i = 0, since_sync = 0;
    bool pending = false;  // fast-path work not yet checked
    // Check queued work; on a capacity overflow, grow and rewind to the
    // failing gate (its input buffer is untouched).
    auto checkpoint = [&](bool* rewound) -> int {
        *rewound = false;
        int st = 0, fail = 0;
        int r = read_status_size(s, &st, &fail);
        if (r) return r;
        since_sync = 0;
        pending = false;
        if (st == 0) return PL_OK;
        if (st != PL_ERR_CAPACITY) return record_status(st, "propagate: device check");
        s->cur = in_buf[fail];
        s->cls = 2;
        i64 m = 0, k[2] = {0, 0};
        PL_CUDA_TRY(cudaMemcpyAsync(&m, s->d_size + s->cur, sizeof(i64), cudaMemcpyDeviceToHost,
                                    s->st));
        PL_CUDA_TRY(cudaMemcpyAsync(k, s->d_k, sizeof(k), cudaMemcpyDeviceToHost, s->st));
        PL_CUDA_TRY(cudaStreamSynchronize(s->st));
        r = clear_status(s);
        if (r) return r;
        r = state_grow(s, 2 * std::max<i64>(m + k[0] + k[1], 2 * m));
        if (r) return r;
        i = (size_t)fail;
        *rewound = true;
        return PL_OK;
    };
    while (i < ops.size()) {
        if (s->cancel && *s->cancel) {
            // drain what is queued (a capacity rewind leaves the failing
            // gate's input in place), then stop between gates
            bool rw = false;
            rc = checkpoint(&rw);
            if (rc) return rc;
            return record_status(PL_ERR_CANCELLED, "propagate: cancelled");
        }
        const Op& op = ops[i];
        bool rewound = false;
        if (op.kind == 2) {
            // a bulk Clifford gate: a bijection of the strings, in place
            in_buf[i] = s->cur;
            if (s->cls == 2) s->cls = 1;
            const bool two = op.gate >= PL_GATE_CNOT;
            const int q2 = two ? op.b : op.a;
            u64 tb;
            u32 ts;
            gate_table(op.gate, &tb, &ts);
            k_clifford<AS><<<grid_persistent(8), 256, 0, s->st>>>(
                s->S[s->cur], s->d_size + s->cur, op.a / 64, 1ull << (op.a % 64), q2 / 64,
                1ull << (q2 % 64), two ? 1 : 0, tb, ts, s->d_status), pl::note_launch();
            pending = true;
            ++since_sync;
            ++i;
        } else if (op.kind == 1) {
            // consecutive CNOTs (one brickwork layer) in one pass
            size_t j = i;
            while (j < ops.size() && ops[j].kind == 1) in_buf[j++] = s->cur;
            if (s->cls == 2) s->cls = 1;
            cudaEvent_t e0 = timed_begin(s->st);
            k_cnot_layer<AS><<<grid_persistent(8), 256, 0, s->st>>>(
                s->S[s->cur], s->d_size + s->cur, s->d_pairs + 2 * i, (int)(j - i), s->d_status),
                pl::note_launch();
            timed_end(e0, s->st, "k_cnot_layer", 0ull);
            pending = true;
            since_sync += j - i;
            i = j;
        } else {
            const int r = op.a;
            const bool fast_ok = singles[r] && (s->cls == 2 || s->cls == 1);
            if (fast_ok && s->cls == 1 && modes[r] != kSkip) {
                // the state must be canonical (sorted) before the merge path
                rc = checkpoint(&rewound);
                if (rc) return rc;
                if (rewound) continue;
                rc = state_canonical_sort(s);
                if (rc) return rc;
            }
            if (fast_ok && s->cls == 2) {
                size_t j = i;
                while (j < ops.size() && ops[j].kind == 0 && singles[ops[j].a]) ++j;
                const int len = (int)(j - i);
                if (s->use_graphs && !trimming && len >= kGraphMin && !timing_enabled()) {
                    for (int q = 0; q < len; ++q) in_buf[i + q] = s->cur ^ (q & 1);
                    rc = rotation_graph<AS>(s, (int)i, len, tr);
                    if (rc) return rc;
                    since_sync += len;
                    i = j;
                } else {
                    in_buf[i] = s->cur;
                    if (modes[r] == kNegate) {
                        k_negate<AS><<<grid_persistent(8), 256, 0, s->st>>>(
                            s->S[s->cur], s->d_size + s->cur, gates[r], 1, s->d_status),
                            pl::note_launch();
                    } else if (modes[r] != kSkip) {
                        rc = rotation_chain<AS>(s, s->cur, (int)i, tr, true);
                        if (rc) return rc;
                        s->cur ^= 1;
                    }
                    if (trimming) {
                        rc = trim_state<AS>(s, tr.max_terms, no_protect);
                        if (rc) return rc;
                    }
                    ++i;
                    ++since_sync;
                }
                pending = true;
            } else if (modes[r] == kSkip && s->cls == 2) {
                if (trimming) {
                    in_buf[i] = s->cur;
                    rc = trim_state<AS>(s, tr.max_terms, no_protect);
                    if (rc) return rc;
                    pending = true;
                }
                ++i;
            } else {
                // general path (synchronous)
                rc = checkpoint(&rewound);
                if (rc) return rc;
                if (rewound) continue;
                i64 m_in = 0, k_anti = 0;
                if (s->gate_log && s->d_log && (rc = read_size(s, &m_in))) return rc;
                rc = general_rotation<AS>(s, rots[r], true, tr, &k_anti);
                if (rc) return rc;
                if (s->gate_log && s->d_log) {
                    i64 trip[3] = {m_in, k_anti, 0};
                    if ((rc = read_size(s, &trip[2]))) return rc;
                    PL_CUDA_TRY(cudaMemcpyAsync(s->d_log + 3 * i, trip, sizeof(trip),
                                                cudaMemcpyHostToDevice, s->st));
                    PL_CUDA_TRY(cudaStreamSynchronize(s->st));
                }
                if (trimming) {
                    rc = trim_state<AS>(s, tr.max_terms, no_protect);
                    if (rc) return rc;
                }
                ++i;
            }
        }
        if (pending && (since_sync >= (size_t)kWindow || i == ops.size())) {
            rc = checkpoint(&rewound);
            if (rc) return rc;
        }
    }
    PL_CUDA_TRY(cudaGetLastError());
    return PL_OK;
}

int check_state(pl_state* s) {
    if (!s) return record_status(PL_ERR_INVALID_ARG, "pl_state is NULL");
    return PL_OK;
}

std::vector<Rot> host_rotations(int as, const u64* rx, const u64* rz, const u8* rf,
                                const double* th, i64 n_rot) {
    std::vector<Rot> v((size_t)n_rot);
    for (i64 r = 0; r < n_rot; ++r) {
        v[r].px.resize(as);
        v[r].pz.resize(as);
        for (int k = 0; k < as; ++k) {
            v[r].px[k] = rx[(size_t)k * n_rot + r];
            v[r].pz[k] = rz[(size_t)k * n_rot + r];
        }
        v[r].pf = rf ? rf[r] : 0;
        v[r].theta = th[r];
    }
    return v;
}

}  // namespace
}  // namespace pl

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" int pl_state_create(pl_state** out, int array_size, int64_t capacity_hint,
                               cudaStream_t stream) {
    if (!out || array_size < 1 || array_size > kMaxAS || capacity_hint < 0)
        return record_status(PL_ERR_INVALID_ARG, "pl_state_create");
    pl_state* s = new pl_state();
    s->as = array_size;
    s->st = stream;
    s->ws.st = stream;
    const int rc = state_grow(s, std::max<int64_t>(capacity_hint, 1 << 16));
    if (rc) {
        delete s;
        return rc;
    }
    *out = s;
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_state_destroy(pl_state* s) {
    if (!s) return record_status(PL_OK, nullptr);
    cudaStreamSynchronize(s->st);
    drop_graphs(s);
    if (s->cap_st) cudaStreamDestroy(s->cap_st);
    if (s->mem) dev_free(s->mem, s->st);
    if (s->d_table) dev_free(s->d_table, s->st);
    if (s->d_pairs) dev_free(s->d_pairs, s->st);
    if (s->budget) s->budget->resize(s->held_bytes + s->ws.bytes, 0);
    if (s->ws.ptr) dev_free(s->ws.ptr, s->st);
    s->ws.ptr = nullptr;
    if (s->trim_mem) dev_free(s->trim_mem, s->st);
    if (s->red) dev_free(s->red, s->st);
    if (s->d_log) dev_free(s->d_log, s->st);
    cudaStreamSynchronize(s->st);
    delete s;
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_state_set_option(pl_state* s, int option, int64_t value) {
    int rc = check_state(s);
    if (rc) return rc;
    if (option == PL_OPT_GRAPHS) {
        s->use_graphs = value != 0;
        if (!s->use_graphs) drop_graphs(s);
        return record_status(PL_OK, nullptr);
    }
    if (option == PL_OPT_GATE_LOG) {
        if ((value != 0) != s->gate_log) drop_graphs(s);  // chains with / without the log
        s->gate_log = value != 0;
        return record_status(PL_OK, nullptr);
    }
    return record_status(PL_ERR_INVALID_ARG, "pl_state_set_option: unknown option");
}

extern "C" int pl_state_set_cancel_flag(pl_state* s, const int32_t* flag) {
    int rc = check_state(s);
    if (rc) return rc;
    s->cancel = flag;
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_state_gate_log(pl_state* s, int64_t* sizes, int64_t max_ops, int64_t* n_ops) {
    int rc = check_state(s);
    if (rc) return rc;
    if (!n_ops || max_ops < 0 || (max_ops > 0 && !sizes))
        return record_status(PL_ERR_INVALID_ARG, "pl_state_gate_log");
    *n_ops = s->d_log ? s->log_used : 0;
    const i64 n = std::min<i64>(*n_ops, max_ops);
    if (n > 0) {
        PL_CUDA_TRY(cudaMemcpyAsync(sizes, s->d_log, 24 * (size_t)n, cudaMemcpyDeviceToHost,
                                    s->st));
        PL_CUDA_TRY(cudaStreamSynchronize(s->st));
    }
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_state_memory(pl_state* s, uint64_t* bytes) {
    int rc = check_state(s);
    if (rc) return rc;
    if (!bytes) return record_status(PL_ERR_INVALID_ARG, "pl_state_memory");
    *bytes = s->held_bytes + s->ws.bytes + s->table_bytes + s->pairs_bytes;
    return record_status(PL_OK, nullptr);
}

namespace pl {
PL_SPIN_LIMIT_SETTER(set_spin_limit_propagate)

// Internal hooks of the sharded collate (pl_shard.cu): the current planes of
// a state, and making room for / setting its term count.
int state_planes(pl_state* s, u64** x, u64** z, u8** f, double** v, i64* cap, i64* n) {
    i64 m = 0;
    const int rc = read_size(s, &m);
    if (rc) return rc;
    const Buf& b = s->S[s->cur];
    *x = b.x;
    *z = b.z;
    *f = b.f;
    *v = b.v;
    *cap = b.cap;
    *n = m;
    return PL_OK;
}
int state_reserve(pl_state* s, i64 n) { return n > s->cap ? state_grow(s, n) : PL_OK; }
int state_set_size(pl_state* s, i64 n) {
    PL_CUDA_TRY(cudaMemcpyAsync(s->d_size + s->cur, &n, sizeof(i64), cudaMemcpyHostToDevice,
                                s->st));
    PL_CUDA_TRY(cudaStreamSynchronize(s->st));
    s->cls = 0;
    return PL_OK;
}
cudaStream_t state_stream(pl_state* s) { return s->st; }
int state_array_size(pl_state* s) { return s->as; }

// Internal hooks of the batch executor (pl_batch.cu).
void state_attach_budget(pl_state* s, MemBudget* b) {
    if (s->budget == b) return;
    if (s->budget) s->budget->resize(s->held_bytes + s->ws.bytes, 0);
    s->budget = b;
    if (b) b->resize(0, s->held_bytes + s->ws.bytes);
}
size_t state_held_bytes(pl_state* s) { return s->held_bytes + s->ws.bytes; }
// Give the buffers back (down to the minimum capacity) between jobs.
int state_shrink(pl_state* s) {
    PL_CUDA_TRY(cudaStreamSynchronize(s->st));
    drop_graphs(s);
    const size_t before = s->held_bytes + s->ws.bytes;
    if (s->ws.ptr) dev_free(s->ws.ptr, s->st);
    s->ws.ptr = nullptr;
    s->ws.bytes = 0;
    if (s->mem) dev_free(s->mem, s->st);
    s->mem = nullptr;
    s->cap = 0;
    s->held_bytes = 0;
    if (s->budget) s->budget->resize(before, 0);
    s->cls = 0;
    return state_grow(s, 1 << 16);
}
}  // namespace pl

extern "C" int pl_state_upload(pl_state* s, const uint64_t* x, const uint64_t* z,
                               const uint8_t* flags, const double* val, int64_t n) {
    int rc = check_state(s);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!x || !z || !flags || !val)) || n >= (1ll << 30))
        return record_status(PL_ERR_INVALID_ARG, "pl_state_upload");
    if (n > s->cap) {
        rc = state_grow(s, 2 * n);
        if (rc) return rc;
    }
    const Buf& b = s->S[s->cur];
    if (n > 0) {
        PL_CUDA_TRY(cudaMemcpy2DAsync(b.x, 8 * b.cap, x, 8 * n, 8 * n, s->as,
                                      cudaMemcpyHostToDevice, s->st));
        PL_CUDA_TRY(cudaMemcpy2DAsync(b.z, 8 * b.cap, z, 8 * n, 8 * n, s->as,
                                      cudaMemcpyHostToDevice, s->st));
        PL_CUDA_TRY(cudaMemcpyAsync(b.f, flags, n, cudaMemcpyHostToDevice, s->st));
        PL_CUDA_TRY(cudaMemcpyAsync(b.v, val, 8 * n, cudaMemcpyHostToDevice, s->st));
    }
    i64 nn = n;
    PL_CUDA_TRY(cudaMemcpyAsync(s->d_size + s->cur, &nn, sizeof(i64), cudaMemcpyHostToDevice,
                                s->st));
    PL_CUDA_TRY(cudaMemsetAsync(s->d_status, 0, 2 * sizeof(int), s->st));
    PL_CUDA_TRY(cudaStreamSynchronize(s->st));
    s->cls = 0;
    s->size_hint = n;
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_state_size(pl_state* s, int64_t* n) {
    int rc = check_state(s);
    if (rc) return rc;
    if (!n) return record_status(PL_ERR_INVALID_ARG, "pl_state_size");
    i64 v = 0;
    rc = read_size(s, &v);
    if (rc) return rc;
    *n = v;
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_state_download(pl_state* s, uint64_t* x, uint64_t* z, uint8_t* flags,
                                 double* val, int64_t capacity, int64_t* n_out) {
    int rc = check_state(s);
    if (rc) return rc;
    if (!n_out) return record_status(PL_ERR_INVALID_ARG, "pl_state_download");
    i64 n = 0;
    rc = read_size(s, &n);
    if (rc) return rc;
    *n_out = n;
    if (!x) return record_status(PL_OK, nullptr);
    if (n > capacity || !z || !flags || !val)
        return record_status(PL_ERR_CAPACITY, "pl_state_download: host buffer too small");
    const Buf& b = s->S[s->cur];
    if (n > 0) {
        PL_CUDA_TRY(cudaMemcpy2DAsync(x, 8 * n, b.x, 8 * b.cap, 8 * n, s->as,
                                      cudaMemcpyDeviceToHost, s->st));
        PL_CUDA_TRY(cudaMemcpy2DAsync(z, 8 * n, b.z, 8 * b.cap, 8 * n, s->as,
                                      cudaMemcpyDeviceToHost, s->st));
        PL_CUDA_TRY(cudaMemcpyAsync(flags, b.f, n, cudaMemcpyDeviceToHost, s->st));
        PL_CUDA_TRY(cudaMemcpyAsync(val, b.v, 8 * n, cudaMemcpyDeviceToHost, s->st));
    }
    PL_CUDA_TRY(cudaStreamSynchronize(s->st));
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_state_evolve(pl_state* s, const uint64_t* rot_x, const uint64_t* rot_z,
                               const uint8_t* rot_flags, const double* rot_theta,
                               int64_t n_rot) {
    int rc = check_state(s);
    if (rc) return rc;
    if (n_rot < 0 || (n_rot > 0 && (!rot_x || !rot_z || !rot_theta)))
        return record_status(PL_ERR_INVALID_ARG, "pl_state_evolve");
    const auto rots = host_rotations(s->as, (const u64*)rot_x, (const u64*)rot_z, rot_flags,
                                     rot_theta, n_rot);
    pl_truncation tr{~0ull, 0.0, ~0ull};
    PL_DISPATCH_AS(s->as, for (const Rot& r : rots) {
        double c, sn;
        if (classify(r.theta, &c, &sn) == kSkip) continue;
        rc = general_rotation<AS>(s, r, false, tr);
        if (rc) return rc;
    });
    int st = 0, fail = 0;
    rc = read_status(s, &st, &fail);
    if (rc) return rc;
    if (st) return record_status(st, "pl_state_evolve");
    return record_status(PL_OK, nullptr);
}

static int collate_state_api(pl_state* s, int mode, double cutoff, uint64_t max_weight) {
    int rc = check_state(s);
    if (rc) return rc;
    i64 n = 0;
    rc = read_size(s, &n);
    if (rc) return rc;
    CollateArgs a;
    a.mode = mode;
    a.cutoff = cutoff;
    a.max_weight = max_weight;
    rc = state_collate(s, n, a);
    if (rc) return rc;
    s->cls = mode == kCombine ? 0 : 2;
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_state_canonicalize(pl_state* s) {
    return collate_state_api(s, kCanon, 0.0, ~0ull);
}
extern "C" int pl_state_sort_and_combine(pl_state* s) {
    return collate_state_api(s, kCombine, 0.0, ~0ull);
}
static int trim_api(pl_state* s, uint64_t max_terms, pl_state* keep) {
    int rc = check_state(s);
    if (rc) return rc;
    Protect P{nullptr, nullptr, 0, 0};
    void* prot = nullptr;
    if (keep) {
        rc = check_state(keep);
        if (rc) return rc;
        if (keep->as != s->as) return record_status(PL_ERR_INVALID_ARG, "trim: keep array_size");
        // the protected (x, z) patterns, sorted on the host (the keep set is
        // small: the observable at t = 0 in the reference's use)
        i64 kn = 0;
        rc = read_size(keep, &kn);
        if (rc) return rc;
        if (kn > 0) {
            const int as = s->as;
            std::vector<u64> kx((size_t)as * kn), kz((size_t)as * kn);
            const Buf& b = keep->S[keep->cur];
            PL_CUDA_TRY(cudaMemcpy2DAsync(kx.data(), 8 * kn, b.x, 8 * b.cap, 8 * kn, as,
                                          cudaMemcpyDeviceToHost, keep->st));
            PL_CUDA_TRY(cudaMemcpy2DAsync(kz.data(), 8 * kn, b.z, 8 * b.cap, 8 * kn, as,
                                          cudaMemcpyDeviceToHost, keep->st));
            PL_CUDA_TRY(cudaStreamSynchronize(keep->st));
            std::vector<i64> idx((size_t)kn);
            for (i64 i = 0; i < kn; ++i) idx[(size_t)i] = i;
            auto key_less = [&](i64 a, i64 c) {
                for (int w = 0; w < as; ++w)
                    if (kx[(size_t)w * kn + a] != kx[(size_t)w * kn + c])
                        return kx[(size_t)w * kn + a] < kx[(size_t)w * kn + c];
                for (int w = 0; w < as; ++w)
                    if (kz[(size_t)w * kn + a] != kz[(size_t)w * kn + c])
                        return kz[(size_t)w * kn + a] < kz[(size_t)w * kn + c];
                return false;
            };
            std::sort(idx.begin(), idx.end(), key_less);
            std::vector<u64> sx((size_t)as * kn), sz((size_t)as * kn);
            for (i64 i = 0; i < kn; ++i)
                for (int w = 0; w < as; ++w) {
                    sx[(size_t)w * kn + i] = kx[(size_t)w * kn + idx[(size_t)i]];
                    sz[(size_t)w * kn + i] = kz[(size_t)w * kn + idx[(size_t)i]];
                }
            PL_CUDA_TRY(dev_alloc(&prot, 16 * (size_t)as * kn, s->st));
            u64* px = static_cast<u64*>(prot);
            PL_CUDA_TRY(cudaMemcpyAsync(px, sx.data(), 8 * (size_t)as * kn, cudaMemcpyHostToDevice,
                                        s->st));
            PL_CUDA_TRY(cudaMemcpyAsync(px + (size_t)as * kn, sz.data(), 8 * (size_t)as * kn,
                                        cudaMemcpyHostToDevice, s->st));
            P = Protect{px, px + (size_t)as * kn, kn, kn};
        }
    }
    PL_DISPATCH_AS(s->as, rc = trim_state<AS>(s, max_terms, P));
    if (prot) dev_free(prot, s->st);
    if (rc) return rc;
    int st = 0, fail = 0;
    rc = read_status(s, &st, &fail);
    if (rc) return rc;
    if (st) return record_status(st, "trim");
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_state_trim(pl_state* s, uint64_t max_terms) {
    return trim_api(s, max_terms, nullptr);
}
extern "C" int pl_state_trim_protected(pl_state* s, uint64_t max_terms, pl_state* keep) {
    return trim_api(s, max_terms, keep);
}

extern "C" int pl_state_apply_truncation(pl_state* s, const pl_truncation* o) {
    if (!o) return record_status(PL_ERR_INVALID_ARG, "pl_state_apply_truncation");
    const int rc = collate_state_api(s, kCanon,
                                     o->coefficient_cutoff > 0 ? o->coefficient_cutoff : 0.0,
                                     o->max_weight);
    if (rc || o->max_terms == ~0ull) return rc;
    return trim_api(s, o->max_terms, nullptr);
}

static int filter_state(pl_state* s, double eps, uint64_t max_weight) {
    int rc = check_state(s);
    if (rc) return rc;
    i64 n = 0;
    rc = read_size(s, &n);
    if (rc) return rc;
    const int other = 1 - s->cur;
    PL_CUDA_TRY(cudaMemsetAsync(s->lbA, 0, s->zero_bytes, s->st));
    PL_DISPATCH_AS(s->as, k_filter<AS><<<grid_persistent(4), kPT, 0, s->st>>>(
                              s->S[s->cur], n, s->S[other], eps, max_weight, s->d_size + other,
                              s->lbC, s->ctr + 3, s->d_status), pl::note_launch());
    PL_CUDA_TRY(cudaGetLastError());
    if (n == 0) {
        i64 z = 0;
        PL_CUDA_TRY(cudaMemcpyAsync(s->d_size + other, &z, sizeof(i64), cudaMemcpyHostToDevice,
                                    s->st));
    }
    int st = 0, fail = 0;
    rc = read_status(s, &st, &fail);
    if (rc) return rc;
    if (st) return record_status(st, "filter");
    s->cur = other;
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_state_cutoff(pl_state* s, double eps) {
    return filter_state(s, eps > 0 ? eps : -1.0, ~0ull);
}
extern "C" int pl_state_truncate_weight(pl_state* s, uint64_t max_weight) {
    return filter_state(s, 0.0, max_weight);
}

extern "C" int pl_state_apply_cnot(pl_state* s, int control, int target) {
    int rc = check_state(s);
    if (rc) return rc;
    if (control < 0 || target < 0 || control >= 64 * s->as || target >= 64 * s->as ||
        control == target)
        return record_status(PL_ERR_INVALID_ARG, "pl_state_apply_cnot");
    PL_DISPATCH_AS(s->as, k_cnot_state<AS><<<grid_persistent(8), 256, 0, s->st>>>(
                              s->S[s->cur], s->d_size + s->cur, control / 64,
                              1ull << (control % 64), target / 64, 1ull << (target % 64),
                              s->d_status), pl::note_launch());
    PL_CUDA_TRY(cudaGetLastError());
    if (s->cls == 2) s->cls = 1;
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_state_apply_clifford(pl_state* s, int gate, int q1, int q2) {
    int rc = check_state(s);
    if (rc) return rc;
    const bool two = gate >= PL_GATE_CNOT;
    if (gate < PL_GATE_H || gate > PL_GATE_ISWAP || q1 < 0 || q1 >= 64 * s->as ||
        (two && (q2 < 0 || q2 >= 64 * s->as || q2 == q1)))
        return record_status(PL_ERR_INVALID_ARG, "pl_state_apply_clifford");
    if (!two) q2 = q1;
    u64 tb;
    u32 ts;
    gate_table(gate, &tb, &ts);
    PL_DISPATCH_AS(s->as, k_clifford<AS><<<grid_persistent(8), 256, 0, s->st>>>(
                              s->S[s->cur], s->d_size + s->cur, q1 / 64, 1ull << (q1 % 64),
                              q2 / 64, 1ull << (q2 % 64), two ? 1 : 0, tb, ts, s->d_status),
                          pl::note_launch());
    PL_CUDA_TRY(cudaGetLastError());
    if (s->cls == 2) s->cls = 1;
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_state_apply_rotation_gate(pl_state* s, int axis, int qubit, double angle) {
    int rc = check_state(s);
    if (rc) return rc;
    if (axis < 1 || axis > 3 || qubit < 0 || qubit >= 64 * s->as || !std::isfinite(angle))
        return record_status(PL_ERR_INVALID_ARG, "pl_state_apply_rotation_gate");
    i64 n = 0;
    rc = read_size(s, &n);
    if (rc) return rc;
    if (n == 0) return record_status(PL_OK, nullptr);
    if (2 * n > s->cap) {
        rc = state_grow(s, 2 * n);
        if (rc) return rc;
    }
    const double ch = std::cos(angle / 2), sh = std::sin(angle / 2);
    PL_CUDA_TRY(cudaMemsetAsync(s->lbA, 0, s->zero_bytes, s->st));
    const int other = 1 - s->cur;
    PL_DISPATCH_AS(s->as, k_materialize_rgate<AS><<<grid_persistent(4), kPT, 0, s->st>>>(
                              s->S[s->cur], n, qubit / 64, 1ull << (qubit % 64), axis, ch, sh,
                              s->S[other], s->d_tmp, s->lbA, s->ctr + 0, s->d_status),
                          pl::note_launch());
    i64 total = 0;
    int st[2];
    PL_CUDA_TRY(cudaMemcpyAsync(&total, s->d_tmp, sizeof(i64), cudaMemcpyDeviceToHost, s->st));
    PL_CUDA_TRY(cudaMemcpyAsync(st, s->d_status, sizeof(st), cudaMemcpyDeviceToHost, s->st));
    PL_CUDA_TRY(cudaStreamSynchronize(s->st));
    if (st[0]) return record_status(st[0], "apply_rotation_gate: materialise");
    s->cur = other;
    CollateArgs a;
    a.mode = kCombine;
    rc = state_collate(s, total, a);
    if (rc) return rc;
    s->cls = 0;
    return record_status(PL_OK, nullptr);
}

namespace pl {
namespace {
int ensure_red(pl_state* s) {
    if (!s->red) PL_CUDA_TRY(dev_alloc(reinterpret_cast<void**>(&s->red),
                                       sizeof(double) * (kRedBlocks + 1), s->st));
    return PL_OK;
}

int finish_red(pl_state* s, int exp2, double* result, int use_max = 0) {
    k_sum_partials<<<1, 256, 0, s->st>>>(s->red, kRedBlocks, exp2, s->red + kRedBlocks, use_max),
        pl::note_launch();
    PL_CUDA_TRY(cudaMemcpyAsync(result, s->red + kRedBlocks, sizeof(double),
                                cudaMemcpyDeviceToHost, s->st));
    PL_CUDA_TRY(cudaStreamSynchronize(s->st));
    return record_status(PL_OK, nullptr);
}

int reduce_state(pl_state* s, const RedArgs& R, int exp2, double* result) {
    int rc = ensure_red(s);
    if (rc) return rc;
    PL_DISPATCH_AS(s->as, k_reduce_terms<AS><<<kRedBlocks, 256, 0, s->st>>>(
                              s->S[s->cur], s->d_size + s->cur, R, s->red),
                          pl::note_launch());
    return finish_red(s, exp2, result, R.kind == kRedMaxAbs ? 1 : 0);
}
}  // namespace
}  // namespace pl

extern "C" int pl_state_basis_state_expectation(pl_state* s, const uint64_t* bit_words,
                                                double* result) {
    int rc = check_state(s);
    if (rc) return rc;
    if (!bit_words || !result)
        return record_status(PL_ERR_INVALID_ARG, "pl_state_basis_state_expectation");
    RedArgs R{};
    R.kind = kRedBasis;
    for (int k = 0; k < s->as; ++k) R.bits[k] = bit_words[k];
    return reduce_state(s, R, 0, result);
}

extern "C" int pl_state_trace(pl_state* s, int num_qubits, double* result) {
    int rc = check_state(s);
    if (rc) return rc;
    if (!result || num_qubits < 0 || num_qubits > 64 * s->as)
        return record_status(PL_ERR_INVALID_ARG, "pl_state_trace");
    RedArgs R{};
    R.kind = kRedTrace;
    return reduce_state(s, R, num_qubits, result);
}

extern "C" int pl_state_frobenius_norm2(pl_state* s, double* result) {
    int rc = check_state(s);
    if (rc) return rc;
    if (!result) return record_status(PL_ERR_INVALID_ARG, "pl_state_frobenius_norm2");
    RedArgs R{};
    R.kind = kRedFrob;
    return reduce_state(s, R, 0, result);
}

// The magnitude statistics the global trim of a sharded sum needs
// (MpiPauliSum.h:187-210): how many |c| >= threshold, and the largest |c|.
extern "C" int pl_state_count_above(pl_state* s, double threshold, int64_t* count) {
    int rc = check_state(s);
    if (rc) return rc;
    if (!count) return record_status(PL_ERR_INVALID_ARG, "pl_state_count_above");
    RedArgs R{};
    R.kind = kRedCountAbove;
    R.threshold = threshold;
    double r = 0.0;
    rc = reduce_state(s, R, 0, &r);
    *count = (int64_t)r;
    return rc;
}

extern "C" int pl_state_max_abs(pl_state* s, double* result) {
    int rc = check_state(s);
    if (rc) return rc;
    if (!result) return record_status(PL_ERR_INVALID_ARG, "pl_state_max_abs");
    RedArgs R{};
    R.kind = kRedMaxAbs;
    return reduce_state(s, R, 0, result);
}

extern "C" int pl_state_lookup(pl_state* s, const uint64_t* x, const uint64_t* z,
                               uint8_t flags, double* result) {
    int rc = check_state(s);
    if (rc) return rc;
    if (!x || !z || !result) return record_status(PL_ERR_INVALID_ARG, "pl_state_lookup");
    RedArgs R{};
    R.kind = kRedLookup;
    R.qf = flags & 3u;
    for (int k = 0; k < s->as; ++k) {
        R.qx[k] = x[k];
        R.qz[k] = z[k];
    }
    return reduce_state(s, R, 0, result);
}

extern "C" int pl_state_trace_product(pl_state* a, pl_state* b, int num_qubits,
                                      double* result) {
    int rc = check_state(a);
    if (rc) return rc;
    if ((rc = check_state(b))) return rc;
    if (!result || a->as != b->as || num_qubits < 0 || num_qubits > 64 * a->as)
        return record_status(PL_ERR_INVALID_ARG, "pl_state_trace_product");
    if (b->st != a->st) PL_CUDA_TRY(cudaStreamSynchronize(b->st));
    // A's complex weight per pattern: a canonicalized copy
    pl_state* t = nullptr;
    rc = pl_state_create(&t, a->as, 1 << 16, a->st);
    if (rc) return rc;
    rc = pl_state_append(t, a);
    if (!rc) rc = pl_state_canonicalize(t);
    if (!rc) rc = ensure_red(a);
    if (!rc) {
        PL_DISPATCH_AS(a->as, k_trace_join<AS><<<kRedBlocks, 256, 0, a->st>>>(
                                  t->S[t->cur], t->d_size + t->cur, b->S[b->cur],
                                  b->d_size + b->cur, a->red),
                              pl::note_launch());
        rc = finish_red(a, num_qubits, result);
    }
    pl_state_destroy(t);
    return rc ? rc : record_status(PL_OK, nullptr);
}

extern "C" int pl_state_zero_state_expectation(pl_state* s, double* result) {
    int rc = check_state(s);
    if (rc) return rc;
    if (!result) return record_status(PL_ERR_INVALID_ARG, "pl_state_zero_state_expectation");
    i64 n = 0;
    rc = read_size(s, &n);
    if (rc) return rc;
    const Buf& b = s->S[s->cur];
    rc = pl_zero_state_expectation(s->as, (const uint64_t*)b.x, b.f, b.v, n, b.cap,
                                   (double*)s->d_tmp, s->st);
    if (rc) return rc;
    PL_CUDA_TRY(cudaMemcpyAsync(result, s->d_tmp, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    PL_CUDA_TRY(cudaStreamSynchronize(s->st));
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_propagate(pl_state* s, const uint64_t* rot_x, const uint64_t* rot_z,
                            const uint8_t* rot_flags, const double* rot_theta, int64_t n_rot,
                            const int32_t* ops, int64_t n_ops, const pl_truncation* opts) {
    int rc = check_state(s);
    if (rc) return rc;
    if (!opts || n_rot < 0 || (n_rot > 0 && (!rot_x || !rot_z || !rot_theta)) || n_ops < 0 ||
        (ops && n_ops > 0 && !ops))
        return record_status(PL_ERR_INVALID_ARG, "pl_propagate");
    const auto rots = host_rotations(s->as, (const u64*)rot_x, (const u64*)rot_z, rot_flags,
                                     rot_theta, n_rot);
    // Heisenberg order: walk the circuit backwards.
    std::vector<Op> list;
    if (ops) {
        list.reserve((size_t)n_ops);
        for (i64 l = n_ops; l-- > 0;) {
            const int kind = ops[3 * l], a = ops[3 * l + 1], b = ops[3 * l + 2];
            if (kind == PL_OP_ROTATION) {
                if (a < 0 || a >= n_rot)
                    return record_status(PL_ERR_INVALID_ARG, "pl_propagate: rotation index");
            } else if (kind == PL_OP_CNOT) {
                if (a < 0 || b < 0 || a >= 64 * s->as || b >= 64 * s->as || a == b)
                    return record_status(PL_ERR_INVALID_ARG, "pl_propagate: CNOT qubits");
            } else if (kind > PL_OP_CLIFFORD && kind <= PL_OP_CLIFFORD + PL_GATE_ISWAP) {
                const bool two = kind - PL_OP_CLIFFORD >= PL_GATE_CNOT;
                if (a < 0 || a >= 64 * s->as ||
                    (two && (b < 0 || b >= 64 * s->as || a == b)))
                    return record_status(PL_ERR_INVALID_ARG, "pl_propagate: gate qubits");
            } else {
                return record_status(PL_ERR_INVALID_ARG, "pl_propagate: op kind");
            }
            if (kind >= PL_OP_CLIFFORD)
                list.push_back(Op{2, a, b, kind - PL_OP_CLIFFORD});
            else
                list.push_back(Op{kind == PL_OP_CNOT ? 1 : 0, a, b, 0});
        }
    } else {
        for (i64 l = n_rot; l-- > 0;) list.push_back(Op{0, (int)l, 0, 0});
    }
    PL_DISPATCH_AS(s->as, rc = run_ops<AS>(s, rots, list, *opts));
    if (rc) return rc;
    int st = 0, fail = 0;
    rc = read_status(s, &st, &fail);
    if (rc) return rc;
    if (st) return record_status(st, "pl_propagate");
    return record_status(PL_OK, nullptr);
}

// ---------------------------------------------------------------------------
// Algebra on device-resident states.
// ---------------------------------------------------------------------------
extern "C" int pl_state_multiply(pl_state* lhs, pl_state* rhs) {
    int rc = check_state(lhs);
    if (rc) return rc;
    rc = check_state(rhs);
    if (rc) return rc;
    if (lhs->as != rhs->as) return record_status(PL_ERR_INVALID_ARG, "pl_state_multiply: AS");
    i64 n = 0, m = 0;
    rc = read_size(lhs, &n);
    if (rc) return rc;
    rc = read_size(rhs, &m);
    if (rc) return rc;
    if (n > 0 && m > ((1ll << 30) - 1) / n)
        return record_status(PL_ERR_INVALID_ARG, "pl_state_multiply: n*m must be < 2^30");
    if (rhs->st != lhs->st) PL_CUDA_TRY(cudaStreamSynchronize(rhs->st));
    if (n * m > lhs->cap) {
        rc = state_grow(lhs, n * m);
        if (rc) return rc;
    }
    const Buf& a = lhs->S[lhs->cur];
    const Buf& b = rhs->S[rhs->cur];
    const int other = 1 - lhs->cur;
    const Buf& o = lhs->S[other];
    rc = multiply_impl(lhs->as, a.x, a.z, a.f, a.v, n, a.cap, b.x, b.z, b.f, b.v, m, b.cap, o.x,
                       o.z, o.f, o.v, o.cap, lhs->st);
    if (rc) return rc;
    const i64 nm = n * m;
    PL_CUDA_TRY(cudaMemcpyAsync(lhs->d_size + other, &nm, sizeof(i64), cudaMemcpyHostToDevice,
                                lhs->st));
    PL_CUDA_TRY(cudaStreamSynchronize(lhs->st));
    lhs->cur = other;
    lhs->cls = 0;
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_state_multiply_canonicalize(pl_state* lhs, pl_state* rhs) {
    int rc = check_state(lhs);
    if (rc) return rc;
    rc = check_state(rhs);
    if (rc) return rc;
    if (lhs->as != rhs->as)
        return record_status(PL_ERR_INVALID_ARG, "pl_state_multiply_canonicalize: AS");
    i64 n = 0, m = 0;
    rc = read_size(lhs, &n);
    if (rc) return rc;
    rc = read_size(rhs, &m);
    if (rc) return rc;
    if (rhs->st != lhs->st) PL_CUDA_TRY(cudaStreamSynchronize(rhs->st));
    rc = lhs->ws.ensure(multiply_collate_ws_bytes(lhs->as, n, m));
    if (rc) return rc;
    for (int attempt = 0; attempt < 2; ++attempt) {
        const Buf& a = lhs->S[lhs->cur];
        const Buf& b = rhs->S[rhs->cur];
        const int other = 1 - lhs->cur;
        CollateArgs args;
        args.mode = kCanon;
        i64 cnt = 0;
        rc = multiply_collate(lhs->as, view_of(a, n), view_of(b, m), out_of(lhs->S[other]), args,
                              &cnt, lhs->ws.ptr, lhs->ws.bytes, lhs->st);
        if (rc == PL_ERR_CAPACITY && attempt == 0) {
            rc = state_grow(lhs, cnt);
            if (rc) return rc;
            continue;
        }
        if (rc) return rc;
        PL_CUDA_TRY(cudaMemcpyAsync(lhs->d_size + other, &cnt, sizeof(i64),
                                    cudaMemcpyHostToDevice, lhs->st));
        PL_CUDA_TRY(cudaStreamSynchronize(lhs->st));
        lhs->cur = other;
        lhs->cls = 2;
        return record_status(PL_OK, nullptr);
    }
    return record_status(PL_ERR_INTERNAL, "pl_state_multiply_canonicalize");
}

// dst := dst followed by src's terms (PauliSum::add without the merge,
// PauliSumCore.h:210-237); `+=` is this then pl_state_sort_and_combine.
extern "C" int pl_state_append(pl_state* dst, pl_state* src) {
    int rc = check_state(dst);
    if (rc) return rc;
    if ((rc = check_state(src))) return rc;
    if (dst == src || dst->as != src->as)
        return record_status(PL_ERR_INVALID_ARG, "pl_state_append: operands");
    i64 n = 0, m = 0;
    if ((rc = read_size(dst, &n)) || (rc = read_size(src, &m))) return rc;
    if (src->st != dst->st) PL_CUDA_TRY(cudaStreamSynchronize(src->st));
    if (n + m >= (1ll << 30)) return record_status(PL_ERR_INVALID_ARG, "pl_state_append: size");
    if (n + m > dst->cap) {
        rc = state_grow(dst, n + m);
        if (rc) return rc;
    }
    const Buf& d = dst->S[dst->cur];
    const Buf& b = src->S[src->cur];
    if (m > 0) {
        PL_CUDA_TRY(cudaMemcpy2DAsync(d.x + n, 8 * d.cap, b.x, 8 * b.cap, 8 * m, dst->as,
                                      cudaMemcpyDeviceToDevice, dst->st));
        PL_CUDA_TRY(cudaMemcpy2DAsync(d.z + n, 8 * d.cap, b.z, 8 * b.cap, 8 * m, dst->as,
                                      cudaMemcpyDeviceToDevice, dst->st));
        PL_CUDA_TRY(cudaMemcpyAsync(d.f + n, b.f, m, cudaMemcpyDeviceToDevice, dst->st));
        PL_CUDA_TRY(cudaMemcpyAsync(d.v + n, b.v, 8 * m, cudaMemcpyDeviceToDevice, dst->st));
    }
    const i64 nm = n + m;
    PL_CUDA_TRY(cudaMemcpyAsync(dst->d_size + dst->cur, &nm, sizeof(i64), cudaMemcpyHostToDevice,
                                dst->st));
    PL_CUDA_TRY(cudaStreamSynchronize(dst->st));
    dst->cls = 0;
    return record_status(PL_OK, nullptr);
}

extern "C" int pl_state_commutator(pl_state* out, pl_state* a, pl_state* b, int multiply_by_i) {
    int rc = check_state(out);
    if (rc) return rc;
    if ((rc = check_state(a)) || (rc = check_state(b))) return rc;
    if (out == a || out == b || a->as != b->as || out->as != a->as)
        return record_status(PL_ERR_INVALID_ARG, "pl_state_commutator: operands");
    i64 n = 0, m = 0;
    if ((rc = read_size(a, &n)) || (rc = read_size(b, &m))) return rc;
    if (a->st != out->st) PL_CUDA_TRY(cudaStreamSynchronize(a->st));
    if (b->st != out->st) PL_CUDA_TRY(cudaStreamSynchronize(b->st));
    for (int attempt = 0; attempt < 2; ++attempt) {
        const Buf& A = a->S[a->cur];
        const Buf& B = b->S[b->cur];
        Buf& O = out->S[out->cur];
        PL_CUDA_TRY(cudaMemsetAsync(out->d_tmp, 0, sizeof(i64), out->st));
        rc = commutator_impl(out->as, multiply_by_i ? 1 : 0, A.x, A.z, A.f, A.v, n, A.cap, B.x,
                             B.z, B.f, B.v, m, B.cap, O.x, O.z, O.f, O.v, O.cap,
                             (unsigned long long*)out->d_tmp, true, out->st);
        i64 cnt = 0;
        PL_CUDA_TRY(cudaMemcpyAsync(&cnt, out->d_tmp, sizeof(i64), cudaMemcpyDeviceToHost,
                                    out->st));
        PL_CUDA_TRY(cudaStreamSynchronize(out->st));
        if (rc == PL_ERR_CAPACITY && attempt == 0) {
            rc = state_grow(out, cnt);
            if (rc) return rc;
            continue;
        }
        if (rc) return rc;
        PL_CUDA_TRY(cudaMemcpyAsync(out->d_size + out->cur, &cnt, sizeof(i64),
                                    cudaMemcpyHostToDevice, out->st));
        PL_CUDA_TRY(cudaStreamSynchronize(out->st));
        out->cls = 0;
        return record_status(PL_OK, nullptr);
    }
    return record_status(PL_ERR_INTERNAL, "pl_state_commutator");
}
