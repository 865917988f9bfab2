// pl_collate.cu -- the collate engine: canonicalize / sort_and_combine /
// cutoff / truncate_weight, and the fused product + canonicalize.
//
// Reference semantics (PauLIB):
//   sort_and_combine  PauliSumOperations.h:369-461  stable sort on the key
//                     x[0..AS) < z[0..AS) < flags (u64 lexicographic), each
//                     run of equal keys summed left to right from 0.0.
//   canonicalize      PauliSumUtils.h:315-328  fold sign into value, then
//                     sort_and_combine, then drop value == 0.
//   cutoff / weight   PauliSumUtils.h:378-393  order-preserving filters.
//
// B200 design:
//   1. Key analysis: OR/AND masks of every key field -> the bits that vary.
//      The key is re-packed into only its varying bit ranges (order
//      preserving, because constant bits never decide a comparison), so
//      config-sized sums sort on 41-bit keys instead of 129-bit ones.
//   2. Onesweep LSD radix sort of (packed key chunk, u32 payload) pairs with
//      digits of <= 8 bits: one up-front histogram, then ONE kernel per
//      digit pass (match_any warp ranking, decoupled look-back across
//      tiles, shared-memory staged scatter).  The payload is the input index
//      (31 bits) plus the sign bit, so values are fetched once at the end.
//      LSD radix sort is stable, hence equal keys stay in index order.
//   3. Segment pass: heads of equal-key runs get dense segment ids (look-back
//      scan); runs of <= 32 terms are summed left to right by one thread --
//      bit-identical to the reference's order; longer runs are summed by a
//      CTA with a fixed-order reduction.
//   4. Emit pass: keep-filter (zero / cutoff / weight) + look-back compaction
//      writes the output planes in sorted order.
// Every cross-tile wait is bounded (kSpinLimit) and reports PL_ERR_TIMEOUT.

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "pl_collate.cuh"

namespace pl {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;    // 4096 terms per segment / emit tile
constexpr int kRItems = 8;
constexpr int kRTile = kThreads * kRItems;  // 2048 keys per radix tile
constexpr int kRadix = 256;
constexpr int kWarps = kThreads / 32;
constexpr u32 kIdxMask = 0x7fffffffu;
constexpr u32 kSentinel = 0xffffffffu;
constexpr int kMaxFields = 2 * kMaxAS + 1;
constexpr int kMaxPasses = 72;
constexpr int kShortSeg = 32;
constexpr u32 kFlagAgg = 1u << 30;
constexpr u32 kFlagPre = 2u << 30;
constexpr u32 kCountMask = (1u << 30) - 1;

// ---------------------------------------------------------------------------
// Key layout: field f < AS is x word f, AS <= f < 2AS is z word f-AS, field
// 2AS is the flags value (mode dependent).  Field f contributes bits
// [lo, lo+width) at offset off of the packed key, x[0] most significant.
// ---------------------------------------------------------------------------
struct KeyLayout {
    int lo[kMaxFields];
    int width[kMaxFields];
    int off[kMaxFields];
    int total_bits;
    int nchunks;
    u64 seg_mask0;  // chunk-0 mask for segment equality (drops the sign bit in kProp)
    u64 cbits[kMaxFields];  // values of the bits that do not vary
};

struct PassPlan {
    int npasses;
    int chunk[kMaxPasses];
    int shift[kMaxPasses];
    int bits[kMaxPasses];
    int first[kMaxAS * 2 + 2];  // first pass index of chunk c; first[nchunks] = npasses
};

__device__ __forceinline__ u32 flags_field(u32 f, int mode) {
    if (mode == kCanon) return f & 1u;
    if (mode == kCombine) return f & 3u;
    return ((f & 1u) << 1) | ((f >> 1) & 1u);  // kProp: phase, then sign
}

__device__ __forceinline__ u64 place_bits(u64 v, int s) {
    if (s >= 64 || s <= -64) return 0ull;
    return s >= 0 ? (v << s) : (v >> (-s));
}

template <int AS>
__device__ __forceinline__ u64 pack_chunk(const KeyLayout& L, const u64* xw, const u64* zw,
                                          u32 fv, int c) {
    u64 r = 0;
    const int base = 64 * c;
#pragma unroll
    for (int f = 0; f < 2 * AS + 1; ++f) {
        const int w = L.width[f];
        if (w == 0) continue;
        const u64 word = f < AS ? xw[f] : (f < 2 * AS ? zw[f - AS] : (u64)fv);
        const u64 m = w >= 64 ? ~0ull : ((1ull << w) - 1ull);
        r |= place_bits((word >> L.lo[f]) & m, L.off[f] - base);
    }
    return r;
}

// Inverse of pack_chunk for single-chunk layouts: the full key of a term
// from its packed key and the constant bits.
template <int AS>
__device__ __forceinline__ void unpack_key(const KeyLayout& L, u64 packed, u64* xw, u64* zw,
                                           u32& fv) {
#pragma unroll
    for (int f = 0; f < 2 * AS + 1; ++f) {
        const int w = L.width[f];
        u64 word = L.cbits[f];
        if (w) {
            const u64 m = w >= 64 ? ~0ull : ((1ull << w) - 1ull);
            const u64 v = (packed >> L.off[f]) & m;
            word = (word & ~(m << L.lo[f])) | (v << L.lo[f]);
        }
        if (f < AS) xw[f] = word;
        else if (f < 2 * AS) zw[f - AS] = word;
        else fv = (u32)word;
    }
}

// Output flags byte from the flags key field.
__device__ __forceinline__ u32 out_flags(u32 fv, int mode) {
    if (mode == kCombine) return fv & 3u;
    if (mode == kCanon) return fv & 1u;
    return (fv >> 1) & 1u;  // kProp: field is phase << 1 | sign
}

// ---------------------------------------------------------------------------
// Term sources: where keys and values of the (virtual) input come from.
// ---------------------------------------------------------------------------
template <int AS>
struct SoASrc {
    const u64* x;
    const u64* z;
    const u8* f;
    const double* v;
    i64 stride;
    __device__ __forceinline__ void key(u32 i, u64* xw, u64* zw, u32& fl) const {
#pragma unroll
        for (int k = 0; k < AS; ++k) {
            xw[k] = __ldg(x + (i64)k * stride + i);
            zw[k] = __ldg(z + (i64)k * stride + i);
        }
        fl = __ldg(f + i);
    }
    __device__ __forceinline__ double value(u32 i) const { return __ldg(v + i); }
};

// Division by a loop-invariant u32 d via a 32-bit magic multiplier
// (round-up method): q = (t + ((p - t) >> 1)) >> s with t = umulhi(p, m).
struct FastDiv {
    u32 d, m, s;
    static FastDiv make(u32 d) {
        FastDiv f{d, 0, 0};
        if (d > 1) {
            int l = 0;
            while ((1ull << l) < d) ++l;
            f.m = (u32)((((unsigned __int128)1 << 32) * ((1ull << l) - d)) / d + 1);
            f.s = (u32)(l - 1);
        }
        return f;
    }
    __device__ __forceinline__ u32 div(u32 p) const {
        if (d == 1) return p;
        const u32 t = __umulhi(p, m);
        return (t + ((p - t) >> 1)) >> s;
    }
};

// Products of the outer product PauliSum::multiply (PauliSumOperations.h:
// 256-306): index p = i*n + j is lhs[j] * rhs[i], value lhs_j * rhs_i.
template <int AS>
struct ProdSrc {
    const u64 *ax, *az, *bx, *bz;
    const u8 *af, *bf;
    const double *av, *bv;
    u32 n, m;
    i64 sa, sb;  // plane strides of the operands
    FastDiv dn;  // division by n
    __device__ __forceinline__ void split(u32 p, u32& i, u32& j) const {
        i = dn.div(p);
        j = p - i * n;
    }
    __device__ __forceinline__ void key(u32 p, u64* xw, u64* zw, u32& fl) const {
        u32 i, j;
        split(p, i, j);
        PhaseAcc acc;
#pragma unroll
        for (int k = 0; k < AS; ++k) {
            const u64 a_x = __ldg(ax + (i64)k * sa + j), a_z = __ldg(az + (i64)k * sa + j);
            const u64 b_x = __ldg(bx + (i64)k * sb + i), b_z = __ldg(bz + (i64)k * sb + i);
            xw[k] = a_x ^ b_x;
            zw[k] = a_z ^ b_z;
            acc.step(a_x, a_z, b_x, b_z);
        }
        fl = acc.phase(__ldg(af + j), __ldg(bf + i));
    }
    __device__ __forceinline__ double value(u32 p) const {
        u32 i, j;
        split(p, i, j);
        return dmul(__ldg(av + j), __ldg(bv + i));
    }
};

// ---------------------------------------------------------------------------
// 1. Key masks: OR and AND of every key field over all terms.
// ---------------------------------------------------------------------------
template <int AS>
__global__ void __launch_bounds__(256) k_masks(SoASrc<AS> src, u32 n, int mode, u64* orm,
                                               u64* andm) {
    u64 o[2 * AS + 1], a[2 * AS + 1];
#pragma unroll
    for (int f = 0; f < 2 * AS + 1; ++f) { o[f] = 0; a[f] = ~0ull; }
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        u64 xw[AS], zw[AS];
        u32 fl;
        src.key(i, xw, zw, fl);
#pragma unroll
        for (int k = 0; k < AS; ++k) {
            o[k] |= xw[k]; a[k] &= xw[k];
            o[AS + k] |= zw[k]; a[AS + k] &= zw[k];
        }
        const u64 fv = flags_field(fl, mode);
        o[2 * AS] |= fv;
        a[2 * AS] &= fv;
    }
#pragma unroll
    for (int f = 0; f < 2 * AS + 1; ++f) {
        for (int s = 16; s > 0; s >>= 1) {
            o[f] |= __shfl_xor_sync(0xffffffffu, o[f], s);
            a[f] &= __shfl_xor_sync(0xffffffffu, a[f], s);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicOr(orm + f, o[f]);
            atomicAnd(andm + f, a[f]);
        }
    }
}

// ---------------------------------------------------------------------------
// 2. Pack: chunk 0 of the packed key + payload (index | sign << 31), all
//    chunk planes when the key spans several chunks, and the digit
//    histograms of chunk 0's passes.
// ---------------------------------------------------------------------------
template <int AS, class Src>
__global__ void __launch_bounds__(256) k_pack(Src src, u32 n, int mode, KeyLayout L,
                                              PassPlan P, u32 count_mask, u64* keys, u32* pay,
                                              u64* planes, u32* hist) {
    __shared__ u32 sh[8 * kRadix];
    const int np0 = P.first[1] - P.first[0];
    for (int i = threadIdx.x; i < np0 * kRadix; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const u32 wstride = gridDim.x * blockDim.x;
    for (u32 w0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; w0 < n; w0 += wstride) {
        const u32 i = w0 + lane;
        const bool valid = i < n;
        u64 k0 = 0;
        if (valid) {
            u64 xw[AS], zw[AS];
            u32 fl;
            src.key(i, xw, zw, fl);
            const u32 fv = flags_field(fl, mode);
            k0 = pack_chunk<AS>(L, xw, zw, fv, 0);
            keys[i] = k0;
            const u32 sign = (mode == kCombine) ? 0u : ((fl >> 1) & 1u);
            pay[i] = i | (sign << 31);
            if (L.nchunks > 1) {
                planes[i] = k0;
                for (int c = 1; c < L.nchunks; ++c)
                    planes[(i64)c * n + i] = pack_chunk<AS>(L, xw, zw, fv, c);
            }
        }
        for (int p = 0; p < np0; ++p) {
            if (!((count_mask >> p) & 1u)) continue;
            const u32 d = valid ? ((u32)(k0 >> P.shift[p]) & ((1u << P.bits[p]) - 1u)) : kSentinel;
            const u32 peers = __match_any_sync(0xffffffffu, d);
            if (valid && lane == __ffs(peers) - 1) atomicAdd(&sh[p * kRadix + d], __popc(peers));
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < np0 * kRadix; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Digit histograms of the operands of a product.  For a digit made only of
// x / z bits, the product's digit is the XOR of the operands' digits
// (x = ax ^ bx, z = az ^ bz), so the histogram over all n*m products is the
// XOR-convolution of the two operand histograms; only digits that include
// the phase bit must be counted product by product.
template <int AS>
__global__ void __launch_bounds__(256) k_operand_hist(SoASrc<AS> src, u32 n, KeyLayout L,
                                                      PassPlan P, u32 conv_mask, u32* h) {
    __shared__ u32 sh[8 * kRadix];
    const int np0 = P.first[1] - P.first[0];
    for (int i = threadIdx.x; i < np0 * kRadix; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        u64 xw[AS], zw[AS];
        u32 fl;
        src.key(i, xw, zw, fl);
        const u64 k0 = pack_chunk<AS>(L, xw, zw, 0u, 0);
        for (int p = 0; p < np0; ++p)
            if ((conv_mask >> p) & 1u)
                atomicAdd(&sh[p * kRadix + ((u32)(k0 >> P.shift[p]) & ((1u << P.bits[p]) - 1u))],
                          1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < np0 * kRadix; i += blockDim.x)
        if (sh[i]) atomicAdd(&h[i], sh[i]);
}

// hist[p][d] = sum_{d1} hA[p][d1] * hB[p][d1 ^ d] for every pass p in conv_mask.
__global__ void __launch_bounds__(256) k_xor_conv(const u32* hA, const u32* hB, PassPlan P,
                                                  u32 conv_mask, u32* hist) {
    const int p = blockIdx.x;
    if (!((conv_mask >> p) & 1u)) return;
    const u32 R = 1u << P.bits[p];
    const u32 d = threadIdx.x;
    if (d >= R) return;
    u32 acc = 0;
    for (u32 d1 = 0; d1 < R; ++d1) acc += hA[p * kRadix + d1] * hB[p * kRadix + (d1 ^ d)];
    hist[p * kRadix + d] = acc;
}

// Chunk c >= 1: bring chunk c of every term into the current order and
// histogram its passes.
__global__ void __launch_bounds__(256) k_gather_chunk(const u64* __restrict__ planes_c,
                                                      const u32* __restrict__ pay, u32 n,
                                                      PassPlan P, int c, u64* keys, u32* hist,
                                                      int* status) {
    __shared__ u32 sh[8 * kRadix];
    const int p0 = P.first[c], np = P.first[c + 1] - P.first[c];
    for (int i = threadIdx.x; i < np * kRadix; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const u32 wstride = gridDim.x * blockDim.x;
    for (u32 w0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; w0 < n; w0 += wstride) {
        const u32 i = w0 + lane;
        bool valid = i < n;
        u64 k = 0;
        if (valid) {
            const u32 src = pay[i] & kIdxMask;
            if (src >= n) {
                raise_status(status, PL_ERR_INTERNAL);
                valid = false;
            } else {
                k = __ldg(planes_c + src);
                keys[i] = k;
            }
        }
        for (int p = 0; p < np; ++p) {
            const u32 d = valid ? ((u32)(k >> P.shift[p0 + p]) & ((1u << P.bits[p0 + p]) - 1u))
                                : kSentinel;
            const u32 peers = __match_any_sync(0xffffffffu, d);
            if (valid && lane == __ffs(peers) - 1) atomicAdd(&sh[p * kRadix + d], __popc(peers));
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < np * kRadix; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[(size_t)p0 * kRadix + i], sh[i]);
}

// Exclusive scan of each pass's 256 bucket counts (one block per pass).
__global__ void __launch_bounds__(256) k_scan_buckets(u32* hist, int first_pass) {
    __shared__ u32 s[kRadix];
    u32* h = hist + (size_t)(first_pass + blockIdx.x) * kRadix;
    const int t = threadIdx.x;
    s[t] = h[t];
    __syncthreads();
    for (int off = 1; off < kRadix; off <<= 1) {
        const u32 v = t >= off ? s[t - off] : 0u;
        __syncthreads();
        s[t] += v;
        __syncthreads();
    }
    h[t] = s[t] - h[t];
}

// Block-wide exclusive scan of one value per thread (256 threads).
__device__ __forceinline__ u32 block_excl_scan(u32 v, u32* s_warp, u32& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u32 inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const u32 t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    u32 wpre = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        const u32 c = s_warp[w];
        wpre += (w < warp) ? c : 0u;
        tot += c;
    }
    total = tot;
    __syncthreads();
    return wpre + inc - v;
}

// Decoupled look-back over per-tile counters (status | count words).
// Publishes this tile's aggregate, walks predecessors four at a time (one
// round trip per window), publishes the inclusive prefix and returns the
// exclusive prefix.  Bounded.
__device__ __forceinline__ u32 lookback(u32* lb, u32 tile, u32 stride, u32 cnt, int* status) {
    if (tile == 0) {
        st_volatile(lb, kFlagPre | cnt);
        return 0;
    }
    u32* mine = lb + (size_t)tile * stride;
    st_volatile(mine, kFlagAgg | cnt);
    u32 excl = 0;
    i64 t = (i64)tile - 1;
    u32 spins = 0;
    while (t >= 0) {
        u32 w[4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
            w[k] = t - k >= 0 ? ld_volatile(lb + (size_t)(t - k) * stride) : kFlagPre;
        int k = 0;
        bool done = false;
        for (; k < 4; ++k) {
            const u32 fl = w[k] >> 30;
            if (fl == 0) break;
            excl += w[k] & kCountMask;
            if (fl == 2) {
                done = true;
                break;
            }
        }
        if (done) break;
        t -= k;
        if (k == 0) {
            if (++spins > kSpinLimit) {
                raise_status(status, PL_ERR_TIMEOUT);
                break;
            }
            if (spins > 64) __nanosleep(64);
        }
    }
    st_volatile(mine, kFlagPre | ((excl + cnt) & kCountMask));
    return excl;
}

// ---------------------------------------------------------------------------
// 3. One onesweep digit pass: stable scatter of (key, payload) by digit
//    bits [shift, shift+bits).
// ---------------------------------------------------------------------------
struct RadixSmem {
    u32 whist[kWarps * kRadix];
    u32 bloc[kRadix];
    u32 gofs[kRadix];
    u32 swarp[kWarps];
    u32 tile;
};

// LAST: the final pass also fetches each term's coefficient from the source
// and writes it in sorted order, so the segment sums read contiguous values.
template <class Src, bool LAST>
__global__ void __launch_bounds__(kThreads, 4)
    k_radix_pass(const u64* __restrict__ kin, const u32* __restrict__ vin, u64* __restrict__ kout,
                 u32* __restrict__ vout, u32 n, int shift, int bits,
                 const u32* __restrict__ bstart, u32* lb, u32* tile_ctr, int* status, Src src,
                 double* __restrict__ val_out) {
    extern __shared__ __align__(16) unsigned char dsm[];
    u64* skeys = reinterpret_cast<u64*>(dsm);
    u32* svals = reinterpret_cast<u32*>(dsm + sizeof(u64) * kRTile);
    __shared__ RadixSmem S;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) S.tile = atomicAdd(tile_ctr, 1u);
    for (int i = tid; i < kWarps * kRadix; i += kThreads) S.whist[i] = 0;
    __syncthreads();
    const u32 tile = S.tile;
    const u32 base = tile * (u32)kRTile;
    const u32 dmask = (1u << bits) - 1u;

    u64 keys[kRItems];
    u32 vals[kRItems];
    u32 rank[kRItems];
    const u32 wbase = base + (u32)warp * (kRItems * 32);
#pragma unroll
    for (int t = 0; t < kRItems; ++t) {
        const u32 idx = wbase + t * 32 + lane;
        if (idx < n) {
            keys[t] = kin[idx];
            vals[t] = vin[idx];
        } else {
            keys[t] = 0;
            vals[t] = kSentinel;
        }
    }
    u32* wh = S.whist + warp * kRadix;
#pragma unroll
    for (int t = 0; t < kRItems; ++t) {
        const bool valid = (wbase + t * 32 + lane) < n;
        const u32 d = valid ? ((u32)(keys[t] >> shift) & dmask) : kSentinel;
        const u32 peers = __match_any_sync(0xffffffffu, d);
        const int leader = __ffs(peers) - 1;
        u32 before = 0;
        if (valid && lane == leader) {
            before = wh[d];
            wh[d] = before + __popc(peers);
        }
        before = __shfl_sync(0xffffffffu, before, leader);
        rank[t] = before + __popc(peers & lanemask_lt());
        __syncwarp();
    }
    __syncthreads();
    // Per-bucket: exclusive prefix over warps, tile count, block offsets.
    const u32 d = tid;
    u32 run = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        const u32 c = S.whist[w * kRadix + d];
        S.whist[w * kRadix + d] = run;
        run += c;
    }
    u32 total;
    const u32 bl = block_excl_scan(run, S.swarp, total);
    S.bloc[d] = bl;
    const u32 excl = lookback(lb + d, tile, kRadix, run, status);
    S.gofs[d] = bstart[d] + excl;
    __syncthreads();
#pragma unroll
    for (int t = 0; t < kRItems; ++t) {
        if (wbase + t * 32 + lane < n) {
            const u32 dd = (u32)(keys[t] >> shift) & dmask;
            const u32 pos = S.bloc[dd] + S.whist[warp * kRadix + dd] + rank[t];
            skeys[pos] = keys[t];
            svals[pos] = vals[t];
        }
    }
    __syncthreads();
    const u32 tile_n = min((u32)kRTile, n - base);
    for (u32 p = tid; p < tile_n; p += kThreads) {
        const u64 k = skeys[p];
        const u32 dd = (u32)(k >> shift) & dmask;
        const u32 g = S.gofs[dd] + (p - S.bloc[dd]);
        if (g < n) {
            const u32 pv = svals[p];
            kout[g] = k;
            vout[g] = pv;
            if (LAST) val_out[g] = src.value(pv & kIdxMask);
        } else {
            raise_status(status, PL_ERR_INTERNAL);
        }
    }
}

constexpr size_t kRadixDynSmem = sizeof(u64) * kRTile + sizeof(u32) * kRTile;

// ---------------------------------------------------------------------------
// 4. Segments: equal-key runs of the sorted order.
// ---------------------------------------------------------------------------
struct SegCtx {
    const u64* keys;     // sorted top chunk
    const u32* pay;      // sorted payloads
    const double* vals;  // coefficients in sorted order
    const u64* planes;   // chunk planes (nchunks > 1)
    u32 n;
    int nchunks;
    u64 seg_mask0;
    int mode;
};

// Segment fold.  A warp owns 1024 consecutive sorted terms, staged in shared
// memory; lane L folds its own 32 terms left to right (32 independent
// chains per warp), and a second, lane-serial phase folds each lane's
// prefix (the tail of the segment carried in from its left neighbour) onto
// that carry.  Every segment is therefore summed in exactly the reference's
// left-to-right order (PauliSumOperations.h:443-455).  The warp that holds a
// segment's head owns it; an owned segment still open at the end of the
// range is continued chunk by chunk (up to kExtChunks) and otherwise handed
// to k_long_segments.  Results go to segval[head], segflag[head] = 1
// (2 = long, pending); non-heads get segflag 0.
constexpr int kFoldWarps = 4;
constexpr int kLaneSpan = 32;
constexpr u32 kFoldSpan = 32u * kLaneSpan;  // 1024 terms per warp
constexpr u32 kFoldSlots = 33u * 32u;       // lane spans padded to 33 slots (no bank conflicts)
constexpr int kExtChunks = 32;              // at most 1024 more
constexpr size_t kFoldWarpSmem = kFoldSlots * (8 + 4 + 1);
constexpr size_t kFoldSmem = ((kFoldWarpSmem + 15) & ~size_t(15)) * kFoldWarps;

__device__ __forceinline__ bool lane_same_key(const SegCtx& C, u32 e, u64 ke, u64 kprev,
                                              u32 pe, u32 pprev) {
    // e and its predecessor, by top chunk (ke, kprev) and payloads (lower chunks)
    const u64 m_top = C.nchunks == 1 ? C.seg_mask0 : ~0ull;
    if (((ke ^ kprev) & m_top) != 0) return false;
    if (C.nchunks == 1) return true;
    const u32 ia = pe & kIdxMask, ib = pprev & kIdxMask;
    for (int c = 0; c < C.nchunks - 1; ++c) {
        const u64 m = c == 0 ? C.seg_mask0 : ~0ull;
        if (((C.planes[(i64)c * C.n + ia] ^ C.planes[(i64)c * C.n + ib]) & m) != 0) return false;
    }
    return true;
}

template <int MODE>
__device__ __forceinline__ void fold_add(double& r0, double& r1, double v, u32 p) {
    const bool neg = (p >> 31) != 0;
    if (MODE == kCanon) r0 = dadd(r0, neg ? -v : v);
    else if (MODE == kCombine) r0 = dadd(r0, v);
    else if (neg) r1 = dadd(r1, v);
    else r0 = dadd(r0, v);
}

template <int MODE>
__device__ __forceinline__ void fold_close(double* segval, u8* segflag, i64 h, double r0,
                                           double r1) {
    segval[h] = MODE == kProp ? dadd(r0, -r1) : r0;
    segflag[h] = 1;
}

template <int MODE>
__global__ void __launch_bounds__(32 * kFoldWarps) k_fold(SegCtx C, double* segval,
                                                          u8* segflag, u32* long_list,
                                                          u32* counters) {
    extern __shared__ __align__(16) unsigned char fsm[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const u32 gwarp = blockIdx.x * kFoldWarps + warp;
    const u32 w0 = gwarp * kFoldSpan;
    if (w0 >= C.n) return;
    const u32 w1 = min(w0 + kFoldSpan, C.n);
    const u32 cnt = w1 - w0;
    unsigned char* base = fsm + ((kFoldWarpSmem + 15) & ~size_t(15)) * warp;
    double* sv = reinterpret_cast<double*>(base);
    u32* sp = reinterpret_cast<u32*>(base + 8 * kFoldSlots);
    u8* sh = base + 12 * kFoldSlots;
    // ---- staging: coalesced loads, head flags, non-head segflag = 0
    u64 ck = 0;
    u32 cp = 0;
    if (w0 > 0) {
        ck = C.keys[w0 - 1];
        cp = C.pay[w0 - 1];
    }
    // 8 chunks of loads in flight per lane, then the head flags of those chunks
    constexpr int kBatch = 8;
    for (u32 c0 = 0; c0 * 32 < cnt; c0 += kBatch) {
        u64 ke[kBatch];
        u32 pe[kBatch];
        double ve[kBatch];
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
            const u32 i = (c0 + b) * 32 + lane;
            const bool valid = i < cnt;
            ke[b] = valid ? C.keys[w0 + i] : 0ull;
            pe[b] = valid ? C.pay[w0 + i] : 0u;
            ve[b] = valid ? C.vals[w0 + i] : 0.0;
        }
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
            const u32 c = c0 + b;
            const u32 i = c * 32 + lane;
            const u32 e = w0 + i;
            u64 kp = __shfl_up_sync(0xffffffffu, ke[b], 1);
            u32 pp = __shfl_up_sync(0xffffffffu, pe[b], 1);
            if (lane == 0) {
                kp = ck;
                pp = cp;
            }
            if (i < cnt) {
                const bool head = (e == 0) || !lane_same_key(C, e, ke[b], kp, pe[b], pp);
                const u32 slot = c * 33 + lane;
                sh[slot] = head;
                sp[slot] = pe[b];
                sv[slot] = ve[b];
                if (!head) segflag[e] = 0;
            }
            ck = __shfl_sync(0xffffffffu, ke[b], 31);
            cp = __shfl_sync(0xffffffffu, pe[b], 31);
        }
    }
    __syncwarp();
    // ---- phase 1: each lane folds the segments that start inside its span
    const u32 a = (u32)lane * kLaneSpan;
    const u32 sa = (u32)lane * 33u;
    const u32 lcnt = cnt > a ? min(cnt - a, (u32)kLaneSpan) : 0u;
    u32 first_head = lcnt;  // prefix length (terms before the lane's first head)
    i64 h = -1;
    double r0 = 0.0, r1 = 0.0;
    for (u32 i = 0; i < lcnt; ++i) {
        if (sh[sa + i]) {
            if (h >= 0) fold_close<MODE>(segval, segflag, h, r0, r1);
            else first_head = i;
            h = (i64)(w0 + a + i);
            r0 = 0.0;
            r1 = 0.0;
        }
        if (h >= 0) fold_add<MODE>(r0, r1, sv[sa + i], sp[sa + i]);
    }
    // ---- phase 2: lane-serial carry of the segment crossing lane borders
    i64 ch = -1;  // head of the carried segment (-1: owned by an earlier warp)
    double c0 = 0.0, c1 = 0.0;
    for (int L = 0; L < 32; ++L) {
        i64 nh = ch;
        double n0 = c0, n1 = c1;
        if (lane == L && lcnt) {
            for (u32 i = 0; i < first_head; ++i) fold_add<MODE>(n0, n1, sv[sa + i], sp[sa + i]);
            if (first_head < lcnt) {
                if (ch >= (i64)w0) fold_close<MODE>(segval, segflag, ch, n0, n1);
                nh = h;
                n0 = r0;
                n1 = r1;
            }
        }
        ch = __shfl_sync(0xffffffffu, nh, L);
        c0 = __shfl_sync(0xffffffffu, n0, L);
        c1 = __shfl_sync(0xffffffffu, n1, L);
    }
    if (ch < (i64)w0) return;  // the open segment belongs to an earlier warp
    if (w1 == C.n) {
        if (lane == 0) fold_close<MODE>(segval, segflag, ch, c0, c1);
        return;
    }
    // ---- extension: continue the owned open segment past the range
    ck = C.keys[w1 - 1];
    cp = C.pay[w1 - 1];
    int ext = 0;
    for (u32 cb = w1;; cb += 32) {
        if (cb >= C.n) {
            if (lane == 0) fold_close<MODE>(segval, segflag, ch, c0, c1);
            return;
        }
        if (++ext > kExtChunks) {
            if (lane == 0) {
                segflag[ch] = 2;
                long_list[atomicAdd(&counters[2], 1u)] = (u32)ch;
            }
            return;
        }
        const u32 e = cb + lane;
        const bool valid = e < C.n;
        const u64 ke = valid ? C.keys[e] : 0ull;
        const u32 pe = valid ? C.pay[e] : 0u;
        const double ve = valid ? C.vals[e] : 0.0;
        u64 kp = __shfl_up_sync(0xffffffffu, ke, 1);
        u32 pp = __shfl_up_sync(0xffffffffu, pe, 1);
        if (lane == 0) {
            kp = ck;
            pp = cp;
        }
        const bool head = valid && !lane_same_key(C, e, ke, kp, pe, pp);
        const u32 hb = __ballot_sync(0xffffffffu, head || !valid);
        const u32 lim = hb ? (u32)(__ffs(hb) - 1) : 32u;
        // the tail lanes [0, lim) continue the segment, in order
        double q0 = c0, q1 = c1;
        for (u32 k = 0; k < lim; ++k) {
            const double vk = __shfl_sync(0xffffffffu, ve, k);
            const u32 pk = __shfl_sync(0xffffffffu, pe, k);
            fold_add<MODE>(q0, q1, vk, pk);
        }
        c0 = q0;
        c1 = q1;
        if (lim < 32) {
            if (lane == 0) fold_close<MODE>(segval, segflag, ch, c0, c1);
            return;
        }
        ck = __shfl_sync(0xffffffffu, ke, 31);
        cp = __shfl_sync(0xffffffffu, pe, 31);
    }
}

// Long runs: one CTA per run.  The run ends at the next term whose segflag
// is set (every head has one after k_fold); thread t sums elements t,
// t+256, ... in order and the 256 partial sums are combined by a fixed
// binary tree -- a deterministic order for a given run.
__global__ void __launch_bounds__(kThreads) k_long_segments(SegCtx C, const u32* long_list,
                                                            const u32* counters, double* segval,
                                                            u8* segflag) {
    __shared__ double s0[kThreads], s1[kThreads];
    __shared__ u32 s_end;
    const u32 nlong = counters[2];
    for (u32 li = blockIdx.x; li < nlong; li += gridDim.x) {
        const u32 b = long_list[li];
        if (threadIdx.x == 0) s_end = C.n;
        __syncthreads();
        // scan 4096 flags per step, 16-byte aligned groups of 16 per thread
        for (u32 base = (b + 1) & ~15u; base < C.n; base += kThreads * 16) {
            u32 mine = C.n;
            const u32 lo = base + threadIdx.x * 16;
            if (lo + 16 <= C.n) {
                const uint4 q = *reinterpret_cast<const uint4*>(segflag + lo);
                const u32 w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    if (mine == C.n && lo + j > b && ((w[j >> 2] >> (8 * (j & 3))) & 0xffu))
                        mine = lo + j;
            } else {
                for (u32 j = 0; j < 16 && lo + j < C.n; ++j)
                    if (lo + j > b && segflag[lo + j]) {
                        mine = lo + j;
                        break;
                    }
            }
            if (mine < C.n) atomicMin(&s_end, mine);
            __syncthreads();
            const bool found = s_end < C.n;
            __syncthreads();
            if (found) break;
        }
        const u32 e = s_end;
        double a0 = 0.0, a1 = 0.0;
        for (u32 t = b + threadIdx.x; t < e; t += kThreads) {
            const u32 p = C.pay[t];
            const double v = C.vals[t];
            const bool neg = (p >> 31) != 0;
            if (C.mode == kCanon) a0 = dadd(a0, neg ? -v : v);
            else if (C.mode == kCombine) a0 = dadd(a0, v);
            else if (neg) a1 = dadd(a1, v);
            else a0 = dadd(a0, v);
        }
        s0[threadIdx.x] = a0;
        s1[threadIdx.x] = a1;
        __syncthreads();
        for (int st = kThreads / 2; st > 0; st >>= 1) {
            if ((int)threadIdx.x < st) {
                s0[threadIdx.x] = dadd(s0[threadIdx.x], s0[threadIdx.x + st]);
                s1[threadIdx.x] = dadd(s1[threadIdx.x], s1[threadIdx.x + st]);
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            segval[b] = C.mode == kProp ? dadd(s0[0], -s1[0]) : s0[0];
            segflag[b] = 1;
        }
        __syncthreads();
    }
}

struct SegSmem {
    u32 swarp[kWarps];
    u32 tile;
    u32 excl;
};

// No digit pass at all (every key equal): values in input order.
template <class Src>
__global__ void __launch_bounds__(256) k_gather_values(Src src, const u32* pay, u32 n,
                                                       double* vals) {
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        vals[i] = src.value(pay[i] & kIdxMask);
}

// ---------------------------------------------------------------------------
// 5. Emit: keep-filter + order-preserving compaction into the output.
// ---------------------------------------------------------------------------
template <int AS, class Src>
__device__ __forceinline__ void emit_key(const Src& src, const KeyLayout& L, u64 packed,
                                         const u32* pay, u32 pos, int mode, u64* xw, u64* zw,
                                         u32& fl) {
    if (L.nchunks == 1) {
        u32 fv;
        unpack_key<AS>(L, packed, xw, zw, fv);
        fl = out_flags(fv, mode);
    } else {
        src.key(pay[pos] & kIdxMask, xw, zw, fl);
        fl = mode == kCombine ? (fl & 3u) : (fl & 1u);
    }
}

template <int AS, class Src>
__global__ void __launch_bounds__(kThreads) k_emit(Src src, KeyLayout L, const u64* keys,
                                                   const u32* pay, const double* segval,
                                                   const u8* segflag, u32 n, u32* counters,
                                                   u32* lb, int mode, double cutoff,
                                                   u64 max_weight, SoAOut out, i64* d_out_count,
                                                   int* status) {
    // Heads (segflag set) that survive the filters are compacted in order.
    // Warp-striped items: coalesced loads; all flags are loaded before any
    // value so the loads overlap.  counters: [3] tile ctr.
    __shared__ SegSmem S;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) S.tile = atomicAdd(&counters[3], 1u);
    __syncthreads();
    const u32 tile = S.tile;
    const u32 wbase = tile * (u32)kTile + (u32)warp * (kItems * 32);
    u32 headmask = 0;
#pragma unroll
    for (int t = 0; t < kItems; ++t) {
        const u32 e = wbase + t * 32 + lane;
        if (e < n && segflag[e]) headmask |= 1u << t;
    }
    double v[kItems];
    u64 kk[kItems];
#pragma unroll
    for (int t = 0; t < kItems; ++t) {
        const bool hd = (headmask >> t) & 1u;
        v[t] = hd ? segval[wbase + t * 32 + lane] : 0.0;
        kk[t] = hd ? keys[wbase + t * 32 + lane] : 0ull;
    }
    u32 keepmask = 0, wcount = 0;
    u32 myoff[kItems];
#pragma unroll
    for (int t = 0; t < kItems; ++t) {
        const u32 e = wbase + t * 32 + lane;
        bool keep = false;
        if ((headmask >> t) & 1u) {
            keep = (mode == kCombine) || (v[t] != 0.0);
            if (cutoff > 0.0) keep = keep && (fabs(v[t]) >= cutoff);
            if (keep && max_weight != ~0ull) {
                u64 xw[AS], zw[AS];
                u32 f;
                emit_key<AS>(src, L, kk[t], pay, e, mode, xw, zw, f);
                u64 w = 0;
#pragma unroll
                for (int k = 0; k < AS; ++k) w += (u64)__popcll(xw[k] | zw[k]);
                keep = w <= max_weight;
            }
        }
        const u32 bal = __ballot_sync(0xffffffffu, keep);
        myoff[t] = wcount + __popc(bal & lanemask_lt());
        wcount += __popc(bal);
        if (keep) keepmask |= 1u << t;
    }
    u32 total;
    const u32 wexcl = block_excl_scan(lane == 0 ? wcount : 0u, S.swarp, total);
    const u32 wpre = __shfl_sync(0xffffffffu, wexcl, 0);
    if (tid == 0) S.excl = lookback(lb, tile, 1, total, status);
    __syncthreads();
    const u32 base_o = S.excl + wpre;
#pragma unroll
    for (int t = 0; t < kItems; ++t) {
        if (!((keepmask >> t) & 1u)) continue;
        const u32 e = wbase + t * 32 + lane;
        const i64 o = (i64)base_o + myoff[t];
        if (o >= out.capacity) {
            raise_status(status, PL_ERR_CAPACITY);
            continue;
        }
        u64 xw[AS], zw[AS];
        u32 f;
        emit_key<AS>(src, L, kk[t], pay, e, mode, xw, zw, f);
#pragma unroll
        for (int k = 0; k < AS; ++k) {
            out.x[(i64)k * out.capacity + o] = xw[k];
            out.z[(i64)k * out.capacity + o] = zw[k];
        }
        out.f[o] = (u8)f;
        out.v[o] = v[t];
    }
    if (tile == gridDim.x - 1 && tid == 0) *d_out_count = (i64)S.excl + total;
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
inline size_t al(size_t b) { return (b + 255) & ~size_t(255); }

struct Carve {
    unsigned char* p;
    size_t left;
    bool ok = true;
    template <class T>
    T* take(size_t count) {
        const size_t b = al(sizeof(T) * (count ? count : 1));
        if (b > left) {
            ok = false;
            return nullptr;
        }
        T* r = reinterpret_cast<T*>(p);
        p += b;
        left -= b;
        return r;
    }
};

int max_chunks(int as) { return (128 * as + 2 + 63) / 64; }

size_t ws_for(int as, i64 n, int nch) {
    const i64 tiles = (n + kTile - 1) / kTile + 1;
    const i64 rtiles = (n + kRTile - 1) / kRTile + 1;
    size_t b = 0;
    b += 2 * al(8 * n) + 2 * al(4 * n);                  // keys, payload (ping-pong)
    b += al(8 * n);                                      // values in sorted order
    b += nch > 1 ? al(8 * (size_t)n * nch) : al(8);     // chunk planes
    b += al(4 * kMaxPasses * kRadix);                    // histograms / bucket starts
    b += al(4 * (size_t)rtiles * kRadix);                // radix look-back (one pass)
    b += al(4 * (n + 1)) + al(8 * n) + al(4 * n);         // seg_start, seg_sum, long list
    b += 2 * al(4 * tiles);                              // segment / emit look-back
    b += al(4 * (128 + 16 * kRadix));                    // counters + operand histograms
    b += 2 * al(8 * kMaxFields) + al(8) + al(4);          // masks, out count, status
    return b + 1024;
}

void build_layout(int as, int mode, const u64* orm, const u64* andm, KeyLayout& L, PassPlan& P) {
    const int nf = 2 * as + 1;
    std::memset(&L, 0, sizeof(L));
    std::memset(&P, 0, sizeof(P));
    for (int f = 0; f < nf; ++f) {
        const u64 var = orm[f] ^ andm[f];
        L.cbits[f] = andm[f];
        if (var == 0) continue;
        const int lo = __builtin_ctzll(var), hi = 63 - __builtin_clzll(var);
        L.lo[f] = lo;
        L.width[f] = hi - lo + 1;
    }
    int off = 0;
    for (int f = nf - 1; f >= 0; --f) {
        L.off[f] = off;
        off += L.width[f];
    }
    L.total_bits = off;
    L.nchunks = off == 0 ? 1 : (off + 63) / 64;
    L.seg_mask0 = ~0ull;
    if (mode == kProp && L.width[nf - 1] > 0 && L.lo[nf - 1] == 0) L.seg_mask0 = ~1ull;
    int np = 0;
    for (int c = 0; c < L.nchunks; ++c) {
        P.first[c] = np;
        const int cw = std::min(64, off - 64 * c);
        if (cw <= 0) continue;
        const int passes = (cw + 7) / 8;
        const int dw = (cw + passes - 1) / passes;
        for (int p = 0; p < passes; ++p) {
            P.chunk[np] = c;
            P.shift[np] = p * dw;
            P.bits[np] = std::min(dw, cw - p * dw);
            ++np;
        }
    }
    P.first[L.nchunks] = np;
    P.npasses = np;
}

struct Bufs {
    u64 *ka, *kb, *planes;
    u32 *pa, *pb, *hist, *lb, *seg_start, *long_list, *lb_seg, *lb_emit, *counters;
    double *seg_sum, *sv;
    u64 *orm, *andm;
    i64* d_count;
    int* d_status;
};

bool carve(void* ws, size_t bytes, i64 n, int nch, Bufs& B) {
    const i64 tiles = (n + kTile - 1) / kTile + 1;
    const i64 rtiles = (n + kRTile - 1) / kRTile + 1;
    Carve c{(unsigned char*)ws, bytes};
    B.ka = c.take<u64>(n);
    B.kb = c.take<u64>(n);
    B.pa = c.take<u32>(n);
    B.pb = c.take<u32>(n);
    B.sv = c.take<double>(n);
    B.planes = c.take<u64>(nch > 1 ? (size_t)n * nch : 1);
    B.hist = c.take<u32>(kMaxPasses * kRadix);
    B.lb = c.take<u32>((size_t)rtiles * kRadix);
    B.seg_start = c.take<u32>(n + 1);
    B.seg_sum = c.take<double>(n);
    B.long_list = c.take<u32>(n);
    B.lb_seg = c.take<u32>(tiles);
    B.lb_emit = c.take<u32>(tiles);
    B.counters = c.take<u32>(128 + 16 * kRadix);
    B.orm = c.take<u64>(kMaxFields);
    B.andm = c.take<u64>(kMaxFields);
    B.d_count = c.take<i64>(1);
    B.d_status = c.take<int>(1);
    return c.ok;
}

// Histograms that can be derived instead of counted: none for a plain sum.
template <int AS>
u32 derive_histograms(const SoASrc<AS>&, const KeyLayout&, const PassPlan&, Bufs&,
                      cudaStream_t) {
    return 0u;
}

// Products: chunk-0 passes free of flags bits come from operand histograms.
template <int AS>
u32 derive_histograms(const ProdSrc<AS>& src, const KeyLayout& L, const PassPlan& P, Bufs& B,
                      cudaStream_t st) {
    const int np0 = P.first[1] - P.first[0];
    const int wf = L.width[2 * AS];  // the flags field occupies packed bits [0, wf)
    u32 mask = 0;
    for (int p = 0; p < np0; ++p)
        if (P.shift[p] >= wf) mask |= 1u << p;
    if (!mask) return 0u;
    u32* hA = B.counters + 128;                   // scratch after the counters
    u32* hB = hA + 8 * kRadix;
    if (cudaMemsetAsync(hA, 0, sizeof(u32) * 16 * kRadix, st) != cudaSuccess) return 0u;
    const SoASrc<AS> a{src.ax, src.az, src.af, src.av, src.sa};
    const SoASrc<AS> b{src.bx, src.bz, src.bf, src.bv, src.sb};
    k_operand_hist<AS><<<grid_for(src.n, 256, 64), 256, 0, st>>>(a, src.n, L, P, mask, hA),
        pl::note_launch();
    k_operand_hist<AS><<<grid_for(src.m, 256, 64), 256, 0, st>>>(b, src.m, L, P, mask, hB),
        pl::note_launch();
    k_xor_conv<<<np0, 256, 0, st>>>(hA, hB, P, mask, B.hist), pl::note_launch();
    return mask;
}

template <int AS, class Src>
int run_collate(const Src& src, u32 n, int mode, const KeyLayout& L, const PassPlan& P,
                const CollateArgs& a, const SoAOut& out, i64* out_count, Bufs& B,
                cudaStream_t st) {
    const u32 tiles = (n + kTile - 1) / kTile;
    const u32 rtiles = (n + kRTile - 1) / kRTile;
    const int nsm = sm_count();
    PL_CUDA_TRY(cudaMemsetAsync(B.hist, 0, sizeof(u32) * kMaxPasses * kRadix, st));
    PL_CUDA_TRY(cudaMemsetAsync(B.counters, 0, sizeof(u32) * (kMaxPasses + 8), st));
    PL_CUDA_TRY(cudaMemsetAsync(B.d_status, 0, sizeof(int), st));
    PL_CUDA_TRY(cudaMemsetAsync(B.d_count, 0, sizeof(i64), st));
    const int gblocks = grid_for(n, 256, nsm * 8);
    cudaEvent_t e0 = timed_begin(st);
    const u32 derived = derive_histograms<AS>(src, L, P, B, st);
    timed_end(e0, st, "k_xor_conv", 0ull);
    e0 = timed_begin(st);
    k_pack<AS, Src><<<gblocks, 256, 0, st>>>(src, n, mode, L, P, ~derived, B.ka, B.pa, B.planes,
                                             B.hist),
        pl::note_launch();
    timed_end(e0, st, "k_pack", 12ull * n);
    u64 *kin = B.ka, *kout = B.kb;
    u32 *vin = B.pa, *vout = B.pb;
    const SoASrc<1> nosrc{nullptr, nullptr, nullptr, nullptr, 0};
    for (int c = 0; c < L.nchunks; ++c) {
        const int p0 = P.first[c], np = P.first[c + 1] - p0;
        if (np == 0) continue;
        if (c > 0) {
            e0 = timed_begin(st);
            k_gather_chunk<<<gblocks, 256, 0, st>>>(B.planes + (size_t)c * n, vin, n, P, c, kin,
                                                    B.hist, B.d_status), pl::note_launch();
            timed_end(e0, st, "k_gather_chunk", 20ull * n);
        }
        k_scan_buckets<<<np, kRadix, 0, st>>>(B.hist, p0), pl::note_launch();
        for (int p = p0; p < p0 + np; ++p) {
            PL_CUDA_TRY(cudaMemsetAsync(B.lb, 0, sizeof(u32) * (size_t)rtiles * kRadix, st));
            cudaEvent_t ev0 = timed_begin(st);
            const bool last = (p == P.npasses - 1);
            if (last)
                k_radix_pass<Src, true><<<rtiles, kThreads, kRadixDynSmem, st>>>(
                    kin, vin, kout, vout, n, P.shift[p], P.bits[p], B.hist + (size_t)p * kRadix,
                    B.lb, B.counters + 8 + p, B.d_status, src, B.sv), pl::note_launch();
            else
                k_radix_pass<SoASrc<1>, false><<<rtiles, kThreads, kRadixDynSmem, st>>>(
                    kin, vin, kout, vout, n, P.shift[p], P.bits[p], B.hist + (size_t)p * kRadix,
                    B.lb, B.counters + 8 + p, B.d_status, nosrc, nullptr), pl::note_launch();
            // algorithmic bytes: read and write one u64 key + one u32 payload per
            // term (+ the u64 coefficient written by the last pass)
            timed_end(ev0, st, "k_radix_pass", 24ull * n + (last ? 8ull * n : 0ull));
            std::swap(kin, kout);
            std::swap(vin, vout);
        }
    }
    if (P.npasses == 0)
        k_gather_values<Src><<<gblocks, 256, 0, st>>>(src, vin, n, B.sv), pl::note_launch();
    SegCtx C{kin, vin, B.sv, B.planes, n, L.nchunks, L.seg_mask0, mode};
    u8* segflag = reinterpret_cast<u8*>(B.seg_start);
    const u32 fold_blocks = (n + kFoldSpan * kFoldWarps - 1) / (kFoldSpan * kFoldWarps);
    PL_CUDA_TRY(cudaFuncSetAttribute(k_fold<kCanon>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kFoldSmem));
    PL_CUDA_TRY(cudaFuncSetAttribute(k_fold<kCombine>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFoldSmem));
    PL_CUDA_TRY(cudaFuncSetAttribute(k_fold<kProp>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kFoldSmem));
    e0 = timed_begin(st);
    if (mode == kCanon)
        k_fold<kCanon><<<fold_blocks, 32 * kFoldWarps, kFoldSmem, st>>>(
            C, B.seg_sum, segflag, B.long_list, B.counters), pl::note_launch();
    else if (mode == kCombine)
        k_fold<kCombine><<<fold_blocks, 32 * kFoldWarps, kFoldSmem, st>>>(
            C, B.seg_sum, segflag, B.long_list, B.counters), pl::note_launch();
    else
        k_fold<kProp><<<fold_blocks, 32 * kFoldWarps, kFoldSmem, st>>>(
            C, B.seg_sum, segflag, B.long_list, B.counters), pl::note_launch();
    timed_end(e0, st, "k_fold", 20ull * n);
    e0 = timed_begin(st);
    k_long_segments<<<nsm * 2, kThreads, 0, st>>>(C, B.long_list, B.counters, B.seg_sum,
                                                  segflag), pl::note_launch();
    timed_end(e0, st, "k_long_segments", 0ull);
    // Emit over the segment count; the grid covers the worst case (n).
    PL_CUDA_TRY(cudaMemsetAsync(B.lb_emit, 0, sizeof(u32) * tiles, st));
    e0 = timed_begin(st);
    k_emit<AS, Src><<<tiles, kThreads, 0, st>>>(src, L, kin, vin, B.seg_sum, segflag, n,
                                                B.counters, B.lb_emit, mode, a.cutoff,
                                                a.max_weight, out, B.d_count, B.d_status),
        pl::note_launch();
    timed_end(e0, st, "k_emit", 0ull);
    PL_CUDA_TRY(cudaGetLastError());
    i64 cnt = 0;
    int dstat = 0;
    PL_CUDA_TRY(cudaMemcpyAsync(&cnt, B.d_count, sizeof(i64), cudaMemcpyDeviceToHost, st));
    PL_CUDA_TRY(cudaMemcpyAsync(&dstat, B.d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    PL_CUDA_TRY(cudaStreamSynchronize(st));
    *out_count = cnt;
    if (dstat != 0) return record_status(dstat, "collate: device-side check");
    return PL_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
int DevArena::ensure(size_t need) {
    if (need <= bytes) return PL_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    if (cudaMalloc(&ptr, need) != cudaSuccess) {
        cudaGetLastError();
        return record_status(PL_ERR_OOM, "workspace allocation");
    }
    bytes = need;
    return PL_OK;
}
DevArena::~DevArena() {
    if (ptr) cudaFree(ptr);
}

size_t collate_ws_bytes(int as, i64 n) { return ws_for(as, n, max_chunks(as)); }

int collate_soa(int as, const SoAView& in, const SoAOut& out, const CollateArgs& a,
                i64* out_count, void* ws, size_t ws_bytes, cudaStream_t st) {
    if (as < 1 || as > kMaxAS || in.n < 0 || in.n >= (i64)kCountMask || !out_count)
        return record_status(PL_ERR_INVALID_ARG, "collate: bad size or array_size");
    if (a.mode != kCanon && a.mode != kCombine && a.mode != kProp)
        return record_status(PL_ERR_INVALID_ARG, "collate: bad mode");
    *out_count = 0;
    if (in.n == 0) return PL_OK;
    if (!in.x || !in.z || !in.f || !in.v || !out.x || !out.z || !out.f || !out.v)
        return record_status(PL_ERR_INVALID_ARG, "collate: null pointer");
    const u32 n = (u32)in.n;
    Bufs B;
    if (!ws || !carve(ws, ws_bytes, n, max_chunks(as), B))
        return record_status(PL_ERR_INVALID_ARG, "collate: workspace too small");
    int rc = PL_OK;
    PL_DISPATCH_AS(as, {
        SoASrc<AS> src{in.x, in.z, in.f, in.v, in.stride};
        std::vector<u64> init_or(kMaxFields, 0ull), init_and(kMaxFields, ~0ull);
        PL_CUDA_TRY(cudaMemcpyAsync(B.orm, init_or.data(), 8 * kMaxFields,
                                    cudaMemcpyHostToDevice, st));
        PL_CUDA_TRY(cudaMemcpyAsync(B.andm, init_and.data(), 8 * kMaxFields,
                                    cudaMemcpyHostToDevice, st));
        k_masks<AS><<<grid_for(n, 256, sm_count() * 4), 256, 0, st>>>(src, n, a.mode, B.orm,
                                                                     B.andm), pl::note_launch();
        u64 hor[kMaxFields], hand[kMaxFields];
        PL_CUDA_TRY(cudaMemcpyAsync(hor, B.orm, 8 * kMaxFields, cudaMemcpyDeviceToHost, st));
        PL_CUDA_TRY(cudaMemcpyAsync(hand, B.andm, 8 * kMaxFields, cudaMemcpyDeviceToHost, st));
        PL_CUDA_TRY(cudaStreamSynchronize(st));
        KeyLayout L;
        PassPlan P;
        build_layout(AS, a.mode, hor, hand, L, P);
        rc = run_collate<AS>(src, n, a.mode, L, P, a, out, out_count, B, st);
    });
    return rc;
}

size_t multiply_collate_ws_bytes(int as, i64 n, i64 m) {
    return ws_for(as, n * m, max_chunks(as));
}

int multiply_collate(int as, const SoAView& lhs, const SoAView& rhs, const SoAOut& out,
                     const CollateArgs& a, i64* out_count, void* ws, size_t ws_bytes,
                     cudaStream_t st) {
    if (as < 1 || as > kMaxAS || lhs.n < 0 || rhs.n < 0 || !out_count)
        return record_status(PL_ERR_INVALID_ARG, "multiply_collate: bad size");
    if (a.mode != kCanon && a.mode != kCombine)
        return record_status(PL_ERR_INVALID_ARG, "multiply_collate: bad mode");
    *out_count = 0;
    const i64 total = lhs.n * rhs.n;
    if (total >= (i64)kCountMask)
        return record_status(PL_ERR_INVALID_ARG, "multiply_collate: n*m must be < 2^30");
    if (total == 0) return PL_OK;
    const u32 n = (u32)total;
    Bufs B;
    if (!ws || !carve(ws, ws_bytes, n, max_chunks(as), B))
        return record_status(PL_ERR_INVALID_ARG, "multiply_collate: workspace too small");
    int rc = PL_OK;
    PL_DISPATCH_AS(as, {
        // Varying bits of a product lie inside OR(lhs) | OR(rhs) word by word;
        // the operand masks give a conservative layout without touching the
        // n*m products.
        std::vector<u64> init_or(kMaxFields, 0ull), init_and(kMaxFields, ~0ull);
        u64 hor[2][kMaxFields], hand[2][kMaxFields];
        const SoAView* ops[2] = {&lhs, &rhs};
        for (int w = 0; w < 2; ++w) {
            SoASrc<AS> s{ops[w]->x, ops[w]->z, ops[w]->f, ops[w]->v, ops[w]->stride};
            PL_CUDA_TRY(cudaMemcpyAsync(B.orm, init_or.data(), 8 * kMaxFields,
                                        cudaMemcpyHostToDevice, st));
            PL_CUDA_TRY(cudaMemcpyAsync(B.andm, init_and.data(), 8 * kMaxFields,
                                        cudaMemcpyHostToDevice, st));
            k_masks<AS><<<grid_for(ops[w]->n, 256, sm_count() * 4), 256, 0, st>>>(
                s, (u32)ops[w]->n, a.mode, B.orm, B.andm), pl::note_launch();
            PL_CUDA_TRY(cudaMemcpyAsync(hor[w], B.orm, 8 * kMaxFields, cudaMemcpyDeviceToHost, st));
            PL_CUDA_TRY(
                cudaMemcpyAsync(hand[w], B.andm, 8 * kMaxFields, cudaMemcpyDeviceToHost, st));
            PL_CUDA_TRY(cudaStreamSynchronize(st));
        }
        u64 por[kMaxFields], pand[kMaxFields];
        for (int f = 0; f < 2 * AS; ++f) {
            por[f] = hor[0][f] | hor[1][f];
            pand[f] = 0;
        }
        por[2 * AS] = a.mode == kCanon ? 1ull : 3ull;  // the phase (and sign) may vary
        pand[2 * AS] = 0;
        KeyLayout L;
        PassPlan P;
        build_layout(AS, a.mode, por, pand, L, P);
        ProdSrc<AS> src{lhs.x, lhs.z, rhs.x,      rhs.z,      lhs.f,      rhs.f,
                        lhs.v, rhs.v, (u32)lhs.n, (u32)rhs.n, lhs.stride, rhs.stride,
                        FastDiv::make((u32)lhs.n)};
        rc = run_collate<AS>(src, n, a.mode, L, P, a, out, out_count, B, st);
    });
    return rc;
}

}  // namespace pl

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" int pl_collate_workspace_size(int array_size, int64_t n, size_t* bytes) {
    if (!bytes || array_size < 1 || array_size > pl::kMaxAS || n < 0)
        return pl::record_status(PL_ERR_INVALID_ARG, "pl_collate_workspace_size");
    *bytes = pl::collate_ws_bytes(array_size, n);
    return pl::record_status(PL_OK, nullptr);
}

extern "C" int pl_collate(int array_size, const uint64_t* x, const uint64_t* z,
                          const uint8_t* flags, const double* val, int64_t n, uint64_t* out_x,
                          uint64_t* out_z, uint8_t* out_flags, double* out_val,
                          int64_t out_capacity, int64_t* out_count, const pl_collate_opts* opts,
                          void* workspace, size_t workspace_bytes, cudaStream_t stream) {
    if (!opts) return pl::record_status(PL_ERR_INVALID_ARG, "pl_collate: opts is NULL");
    pl::CollateArgs a;
    a.mode = opts->mode == PL_COLLATE_SORT_AND_COMBINE ? pl::kCombine : pl::kCanon;
    if (opts->mode != PL_COLLATE_CANONICALIZE && opts->mode != PL_COLLATE_SORT_AND_COMBINE)
        return pl::record_status(PL_ERR_INVALID_ARG, "pl_collate: bad mode");
    a.cutoff = opts->cutoff;
    a.max_weight = opts->max_weight;
    pl::SoAView in{(const pl::u64*)x, (const pl::u64*)z, flags, val, n, n};
    pl::SoAOut out{(pl::u64*)out_x, (pl::u64*)out_z, out_flags, out_val, out_capacity};
    const int rc = pl::collate_soa(array_size, in, out, a, (pl::i64*)out_count, workspace,
                                   workspace_bytes, stream);
    return pl::record_status(rc, rc ? "pl_collate" : nullptr);
}

extern "C" int pl_multiply_collate_workspace_size(int array_size, int64_t n, int64_t m,
                                                  size_t* bytes) {
    if (!bytes || array_size < 1 || array_size > pl::kMaxAS || n < 0 || m < 0)
        return pl::record_status(PL_ERR_INVALID_ARG, "pl_multiply_collate_workspace_size");
    *bytes = pl::multiply_collate_ws_bytes(array_size, n, m);
    return pl::record_status(PL_OK, nullptr);
}

extern "C" int pl_multiply_collate(int array_size, const uint64_t* lhs_x, const uint64_t* lhs_z,
                                   const uint8_t* lhs_flags, const double* lhs_val, int64_t n,
                                   const uint64_t* rhs_x, const uint64_t* rhs_z,
                                   const uint8_t* rhs_flags, const double* rhs_val, int64_t m,
                                   uint64_t* out_x, uint64_t* out_z, uint8_t* out_flags,
                                   double* out_val, int64_t out_capacity, int64_t* out_count,
                                   const pl_collate_opts* opts, void* workspace,
                                   size_t workspace_bytes, cudaStream_t stream) {
    if (!opts) return pl::record_status(PL_ERR_INVALID_ARG, "pl_multiply_collate: opts");
    pl::CollateArgs a;
    if (opts->mode != PL_COLLATE_CANONICALIZE && opts->mode != PL_COLLATE_SORT_AND_COMBINE)
        return pl::record_status(PL_ERR_INVALID_ARG, "pl_multiply_collate: bad mode");
    a.mode = opts->mode == PL_COLLATE_SORT_AND_COMBINE ? pl::kCombine : pl::kCanon;
    a.cutoff = opts->cutoff;
    a.max_weight = opts->max_weight;
    pl::SoAView l{(const pl::u64*)lhs_x, (const pl::u64*)lhs_z, lhs_flags, lhs_val, n, n};
    pl::SoAView r{(const pl::u64*)rhs_x, (const pl::u64*)rhs_z, rhs_flags, rhs_val, m, m};
    pl::SoAOut out{(pl::u64*)out_x, (pl::u64*)out_z, out_flags, out_val, out_capacity};
    const int rc = pl::multiply_collate(array_size, l, r, out, a, (pl::i64*)out_count, workspace,
                                        workspace_bytes, stream);
    return pl::record_status(rc, rc ? "pl_multiply_collate" : nullptr);
}
