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
#include <type_traits>
#include <vector>

#include "pl_collate.cuh"

namespace pl {

namespace {

constexpr int kThreads = 256;
constexpr int kRTileMin = kThreads * 8;  // smallest radix tile (8 keys per thread)
constexpr int kRadix = 256;
constexpr int kWarps = kThreads / 32;
constexpr u32 kIdxMask = 0x7fffffffu;
constexpr u32 kSentinel = 0xffffffffu;
constexpr int kMaxFields = 2 * kMaxAS + 1;
// Digit passes of the widest key: 2 * 64 * kMaxAS x / z bits and the flags
// field, in chunks of 64 bits of up to 8 passes each.
constexpr int kMaxPasses = 8 * ((2 * 64 * kMaxAS + 2 + 63) / 64);
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

// Phase / sign bit planes of index-packed keys: word w holds, for terms
// 32w .. 32w+31, the imaginary bits (x) and the sign bits (y); n/4 bytes in
// all, small enough to stay in L2 for the gathers of the last digit pass.
__device__ __forceinline__ u32 phase_bits(const uint2* phs, u32 i) {
    const uint2 w = phs[i >> 5];
    const u32 b = i & 31u;
    return ((w.x >> b) & 1u) | (((w.y >> b) & 1u) << 1);
}
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
    // Index-packed keys: the phase / sign bits (flags & 3) of term i come from
    // the bit planes k_pack_split stored, the coefficient from the source.
    __device__ __forceinline__ void flags_value(u32 i, const uint2* phs, u32& fl,
                                                double& val) const {
        fl = phase_bits(phs, i);
        val = __ldg(v + i);
    }
    // the term as it is output (the sort key above is the term itself)
    static constexpr bool kVirtualKey = false;
    __device__ __forceinline__ void orig_key(u32 i, u64* xw, u64* zw, u32& fl) const {
        key(i, xw, zw, fl);
    }
};

// ---------------------------------------------------------------------------
// Windowed keys.  When every term's x bits (and z bits) lie in two
// consecutive words and, in each word, within kWinSpan consecutive bits --
// Pauli strings supported on a window of adjacent qubits -- the sort key
// (x[0..AS), z[0..AS), flags) compresses, order preserving, to two virtual
// words per plane:
//   x'[0] = (AS - f) << 22 | win(x[f]),  x'[1] = win(x[f + 1]),  x'[k] = 0
// with f the first nonzero word (f = AS, x'[0] = 0 for x == 0) and win(w) =
// (msb + 1) << (kWinSpan - 1) | the kWinSpan - 1 bits below w's msb.  A
// smaller f means a larger x, and within one f the two words compare as
// their win() values; likewise for z.  The varying-bit analysis then runs
// on the virtual words: for the windowed commutator workload (supports of
// <= 11 qubits on 256) about 80 varying bits instead of 513.  Sort and
// segment detection use the virtual key (it is injective on such terms);
// the emit writes each term's original words, fetched by its index.
// ---------------------------------------------------------------------------
constexpr int kWinSpan = 16;

__device__ __forceinline__ u64 win_word(u64 w) {
    if (!w) return 0;
    const int msb = 63 - __clzll((long long)w);
    const u64 below = msb >= kWinSpan - 1 ? (w >> (msb - (kWinSpan - 1)))
                                          : (w << ((kWinSpan - 1) - msb));
    return ((u64)(msb + 1) << (kWinSpan - 1)) | (below & ((1ull << (kWinSpan - 1)) - 1ull));
}

// Virtual words of one plane; returns false when the plane does not fit the
// window form (nonzero words beyond f + 1, or a word wider than kWinSpan).
template <int AS>
__device__ __forceinline__ bool win_plane(const u64* w, u64* out) {
    int f = AS;
#pragma unroll
    for (int k = AS - 1; k >= 0; --k)
        if (w[k]) f = k;
    bool ok = true;
    u64 w0 = 0, w1 = 0;
#pragma unroll
    for (int k = 0; k < AS; ++k) {
        const u64 v = w[k];
        if (k == f) w0 = v;
        else if (k == f + 1) w1 = v;
        else if (v) ok = false;
        if (v && (63 - __clzll((long long)v)) - (__ffsll((long long)v) - 1) >= kWinSpan)
            ok = false;
    }
    out[0] = f < AS ? ((u64)(AS - f) << 22) | win_word(w0) : 0ull;
#pragma unroll
    for (int k = 1; k < AS; ++k) out[k] = k == 1 ? win_word(w1) : 0ull;
    return ok;
}

template <int AS>
struct WinSrc {
    SoASrc<AS> s;
    __device__ __forceinline__ bool vkey(u32 i, u64* xw, u64* zw, u32& fl) const {
        u64 ox[AS], oz[AS];
        s.key(i, ox, oz, fl);
        const bool a = win_plane<AS>(ox, xw);
        const bool b = win_plane<AS>(oz, zw);
        return a && b;
    }
    __device__ __forceinline__ void key(u32 i, u64* xw, u64* zw, u32& fl) const {
        (void)vkey(i, xw, zw, fl);
    }
    __device__ __forceinline__ double value(u32 i) const { return s.value(i); }
    static constexpr bool kVirtualKey = true;
    __device__ __forceinline__ void orig_key(u32 i, u64* xw, u64* zw, u32& fl) const {
        s.key(i, xw, zw, fl);
    }
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
    // Index-packed keys: the product's phase / sign bits from the bit planes
    // k_pack_split stored, its coefficient from the operands.
    __device__ __forceinline__ void flags_value(u32 p, const uint2* phs, u32& fl,
                                                double& val) const {
        fl = phase_bits(phs, p);
        val = value(p);
    }
    static constexpr bool kVirtualKey = false;
    __device__ __forceinline__ void orig_key(u32 p, u64* xw, u64* zw, u32& fl) const {
        key(p, xw, zw, fl);
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
// Masks of the windowed virtual key (as k_masks) and whether every term fits
// the window form (bad[0] != 0: some term does not).
// OR masks of the x / z words of both operands of a product, one launch and
// no initialisation: blockIdx.y picks the operand, and each block writes its
// partial OR to part[(y * gridDim.x + x) * 2AS + f]; the host ORs the blocks.
template <int AS>
__global__ void __launch_bounds__(256) k_operand_or(SoASrc<AS> a, u32 na, SoASrc<AS> b, u32 nb,
                                                    u64* part) {
    __shared__ u64 sw[kWarps][2 * AS];
    const SoASrc<AS>& src = blockIdx.y ? b : a;
    const u32 n = blockIdx.y ? nb : na;
    u64 o[2 * AS];
#pragma unroll
    for (int f = 0; f < 2 * AS; ++f) o[f] = 0;
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        u64 xw[AS], zw[AS];
        u32 fl;
        src.key(i, xw, zw, fl);
#pragma unroll
        for (int k = 0; k < AS; ++k) {
            o[k] |= xw[k];
            o[AS + k] |= zw[k];
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int f = 0; f < 2 * AS; ++f) {
        for (int d = 16; d > 0; d >>= 1) o[f] |= __shfl_xor_sync(0xffffffffu, o[f], d);
        if (lane == 0) sw[warp][f] = o[f];
    }
    __syncthreads();
    if (threadIdx.x < 2 * AS) {
        u64 v = 0;
        for (int w = 0; w < kWarps; ++w) v |= sw[w][threadIdx.x];
        part[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * (2 * AS) + threadIdx.x] = v;
    }
}

template <int AS>
__global__ void __launch_bounds__(256) k_win_masks(WinSrc<AS> src, u32 n, int mode, u64* orm,
                                                   u64* andm, u32* bad) {
    u64 o[2 * AS + 1], a[2 * AS + 1];
#pragma unroll
    for (int f = 0; f < 2 * AS + 1; ++f) { o[f] = 0; a[f] = ~0ull; }
    bool fits = true;
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        u64 xw[AS], zw[AS];
        u32 fl;
        fits = src.vkey(i, xw, zw, fl) && fits;
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
        for (int s2 = 16; s2 > 0; s2 >>= 1) {
            o[f] |= __shfl_xor_sync(0xffffffffu, o[f], s2);
            a[f] &= __shfl_xor_sync(0xffffffffu, a[f], s2);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicOr(orm + f, o[f]);
            atomicAnd(andm + f, a[f]);
        }
    }
    if (!__all_sync(0xffffffffu, fits) && (threadIdx.x & 31) == 0) atomicOr(bad, 1u);
}

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

// Pack for index-packed keys (kCanonSplit): key = packed (x, z) << index
// bits | index, the phase / sign byte (flags & 3) of each term by index, and
// the digit histograms of the passes not derived from operand histograms.
template <int AS, class Src>
__global__ void __launch_bounds__(256) k_pack_split(Src src, u32 n, KeyLayout L, PassPlan P,
                                                    u32 count_mask, u64* keys, uint2* phs,
                                                    u32* hist) {
    __shared__ u32 sh[8 * kRadix];
    const int np = P.npasses;
    for (int i = threadIdx.x; i < np * kRadix; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const u32 wstride = gridDim.x * blockDim.x;
    for (u32 w0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; w0 < n; w0 += wstride) {
        const u32 i = w0 + lane;
        const bool valid = i < n;
        u64 k0 = 0;
        u32 fl = 0;
        if (valid) {
            u64 xw[AS], zw[AS];
            src.key(i, xw, zw, fl);
            k0 = pack_chunk<AS>(L, xw, zw, 0u, 0) | (u64)i;
            keys[i] = k0;
        }
        {
            const u32 im = __ballot_sync(0xffffffffu, valid && (fl & 1u));
            const u32 sg = __ballot_sync(0xffffffffu, valid && (fl & 2u));
            if (lane == 0) phs[w0 >> 5] = make_uint2(im, sg);
        }
        if (!count_mask) continue;
        for (int p = 0; p < np; ++p) {
            if (!((count_mask >> p) & 1u)) continue;
            const u32 d = valid ? ((u32)(k0 >> P.shift[p]) & ((1u << P.bits[p]) - 1u)) : kSentinel;
            const u32 peers = __match_any_sync(0xffffffffu, d);
            if (valid && lane == __ffs(peers) - 1) atomicAdd(&sh[p * kRadix + d], __popc(peers));
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < np * kRadix; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Pack of a product's index-packed keys when every digit histogram comes
// from the operands (no counting): one block row per rhs term i (its words
// held in registers), lhs terms j across the threads.  Packing is linear
// over XOR (x = ax ^ bx, z = az ^ bz), so the packed key is the XOR of the
// operands' packed keys.  Needs n % 32 == 0 so each warp's 32 products are
// one bit-plane word.
constexpr int kPackPerThread = 8;
//
// opk (optional): the operands' packed keys, lhs then rhs, as k_operand_hist
// stored them -- one load per product instead of re-packing the lhs words.
template <int AS>
__global__ void __launch_bounds__(256) k_pack_split_prod(ProdSrc<AS> src, KeyLayout L, u64* keys,
                                                         uint2* phs, const u64* __restrict__ opk) {
    const u32 i = blockIdx.y;
    const u32 j = blockIdx.x * blockDim.x * kPackPerThread + threadIdx.x;
    u64 bxw[AS], bzw[AS];
#pragma unroll
    for (int k = 0; k < AS; ++k) {
        bxw[k] = __ldg(src.bx + (i64)k * src.sb + i);
        bzw[k] = __ldg(src.bz + (i64)k * src.sb + i);
    }
    const u64 kb = opk ? __ldg(opk + src.n + i) : pack_chunk<AS>(L, bxw, bzw, 0u, 0);
    const u32 bfl = __ldg(src.bf + i);
#pragma unroll
    for (int r = 0; r < kPackPerThread; ++r) {
        const u32 jj = j + (u32)r * blockDim.x;
        if (jj >= src.n) break;  // whole warps: n % 32 == 0
        u64 axw[AS], azw[AS];
        PhaseAcc acc;
#pragma unroll
        for (int k = 0; k < AS; ++k) {
            axw[k] = __ldg(src.ax + (i64)k * src.sa + jj);
            azw[k] = __ldg(src.az + (i64)k * src.sa + jj);
            acc.step(axw[k], azw[k], bxw[k], bzw[k]);
        }
        const u32 fl = acc.phase(__ldg(src.af + jj), bfl);
        const u32 p = i * src.n + jj;
        const u64 ka = opk ? __ldg(opk + jj) : pack_chunk<AS>(L, axw, azw, 0u, 0);
        keys[p] = (ka ^ kb) | (u64)p;
        const u32 im = __ballot_sync(0xffffffffu, (fl & 1u) != 0);
        const u32 sg = __ballot_sync(0xffffffffu, (fl & 2u) != 0);
        if ((threadIdx.x & 31) == 0) phs[p >> 5] = make_uint2(im, sg);
    }
}

// Generic pack unless the product fast path applies.
template <int AS>
bool pack_split_fast(const SoASrc<AS>&, u32, const KeyLayout&, u32, u64*, uint2*, const u64*,
                     cudaStream_t) {
    return false;
}
template <int AS>
bool pack_split_fast(const ProdSrc<AS>& src, u32, const KeyLayout& L, u32 count_mask, u64* keys,
                     uint2* phs, const u64* opk, cudaStream_t st) {
    if (count_mask != 0 || src.n % 32 != 0 || src.m > 65535u) return false;
    const dim3 grid((src.n + 256 * kPackPerThread - 1) / (256 * kPackPerThread), src.m);
    k_pack_split_prod<AS><<<grid, 256, 0, st>>>(src, L, keys, phs, opk), pl::note_launch();
    return true;
}

// Digit histograms of the operands of a product.  For a digit made only of
// x / z bits, the product's digit is the XOR of the operands' digits
// (x = ax ^ bx, z = az ^ bz), so the histogram over all n*m products is the
// XOR-convolution of the two operand histograms; only digits that include
// the phase bit must be counted product by product.
// Both operands in one launch: blockIdx.y 0 counts (src, n) into h, 1 counts
// (src2, n2) into h2.
// With pk set, each term's packed key is stored as well: lhs at pk[0, n),
// rhs at pk[n, n + n2).
// R: bins per pass (256, or 1024 for 10-bit digits); the histograms of pass
// p are at [p * R, p * R + R).
template <int AS, int R = kRadix>
__global__ void __launch_bounds__(256) k_operand_hist(SoASrc<AS> src, u32 n, u32* h,
                                                      SoASrc<AS> src2, u32 n2, u32* h2,
                                                      KeyLayout L, PassPlan P, u32 conv_mask,
                                                      u64* pk) {
    if (blockIdx.y == 1) {
        src = src2;
        if (pk) pk += n;
        n = n2;
        h = h2;
    }
    __shared__ u32 sh[(R == kRadix ? 8 : 4) * R];
    const int np0 = P.first[1] - P.first[0];
    for (int i = threadIdx.x; i < np0 * R; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        u64 xw[AS], zw[AS];
        u32 fl;
        src.key(i, xw, zw, fl);
        const u64 k0 = pack_chunk<AS>(L, xw, zw, 0u, 0);
        if (pk) pk[i] = k0;
        for (int p = 0; p < np0; ++p)
            if ((conv_mask >> p) & 1u)
                atomicAdd(&sh[p * R + ((u32)(k0 >> P.shift[p]) & ((1u << P.bits[p]) - 1u))], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < np0 * R; i += blockDim.x)
        if (sh[i]) atomicAdd(&h[i], sh[i]);
}

__device__ __forceinline__ u32 block_excl_scan(u32 v, u32* s_warp, u32& total);
template <int NW>
__device__ __forceinline__ u32 block_scan_n(u32 v, u32* s_warp, u32& total);

// hist[p][d] = sum_{d1} hA[p][d1] * hB[p][d1 ^ d] for every pass p in conv_mask
// (both operand histograms staged in shared memory).  With scan = 1 every
// pass's histogram is derived, and the block turns it into the pass's
// bucket starts (exclusive prefix) right away, in place of k_scan_buckets.
// NB: bins per pass (256, or 1024 for 10-bit digits), one thread per bin.
template <int NB>
__global__ void __launch_bounds__(NB) k_xor_conv(const u32* hA, const u32* hB, PassPlan P,
                                                 u32 conv_mask, u32* hist, int scan) {
    __shared__ u32 sa[NB], sb[NB], sw[65];
    const int p = blockIdx.x;
    if (!((conv_mask >> p) & 1u)) return;
    const u32 R = 1u << P.bits[p];
    const u32 d = threadIdx.x;
    sa[d] = hA[p * NB + d];
    sb[d] = hB[p * NB + d];
    __syncthreads();
    u32 acc = 0;
    if (d < R)
        for (u32 d1 = 0; d1 < R; ++d1) acc += sa[d1] * sb[d1 ^ d];
    if (!scan) {
        if (d < R) hist[p * NB + d] = acc;
        return;
    }
    u32 total;
    hist[p * NB + d] = block_scan_n<NB / 32>(acc, sw, total);
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

// Decoupled look-back over per-tile counters (status | count words), in two
// halves so a tile can do other work between them: lb_publish posts this
// tile's aggregate (tile 0: its inclusive prefix); lb_walk reads the
// predecessors W at a time (one round trip per window), posts the inclusive
// prefix and returns the exclusive prefix.  Bounded.
__device__ __forceinline__ void lb_publish(u32* lb, u32 tile, u32 stride, u32 cnt) {
    st_volatile(lb + (size_t)tile * stride, (tile == 0 ? kFlagPre : kFlagAgg) | cnt);
}

// hot: polls without progress before each further poll sleeps 64 ns (a
// spinning thread takes issue slots from the warps that do work).
template <int W = 4>
__device__ __forceinline__ u32 lb_walk(u32* lb, u32 tile, u32 stride, u32 cnt, int* status,
                                       u32 hot = 64) {
    if (tile == 0) return 0;
    u32* mine = lb + (size_t)tile * stride;
    u32 excl = 0;
    i64 t = (i64)tile - 1;
    u32 spins = 0;
    while (t >= 0) {
        u32 w[W];
#pragma unroll
        for (int k = 0; k < W; ++k)
            w[k] = t - k >= 0 ? ld_volatile(lb + (size_t)(t - k) * stride) : kFlagPre;
        int k = 0;
        bool done = false;
        for (; k < W; ++k) {
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
            if (++spins > g_spin_limit) {
                raise_status(status, PL_ERR_TIMEOUT);
                break;
            }
            if (spins > hot) __nanosleep(64);
        }
    }
    st_volatile(mine, kFlagPre | ((excl + cnt) & kCountMask));
    return excl;
}

__device__ __forceinline__ u32 lookback(u32* lb, u32 tile, u32 stride, u32 cnt, int* status) {
    lb_publish(lb, tile, stride, cnt);
    return lb_walk<4>(lb, tile, stride, cnt, status);
}

// ---------------------------------------------------------------------------
// 3. One onesweep digit pass: stable scatter of (key, payload) by digit
//    bits [shift, shift+bits).
// ---------------------------------------------------------------------------
// whist[w][d]: per warp w, its digit-d count while ranking, then the tile
// position of its first digit-d key (block offset of d + earlier warps'
// counts).  gofs[d]: global position of the tile's first digit-d key minus
// its tile position, so a key at tile position p goes to gofs[d] + p.
struct RadixSmem {
    u32 whist[kWarps * kRadix];
    u32 gofs[kRadix];
    u32 swarp[kWarps];
    u32 tile;
};

// Bulk prefetch of [p, p + bytes) into L2 (a hint; p 16-byte aligned, bytes a
// multiple of 16).
__device__ __forceinline__ void prefetch_l2(const void* p, u32 bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// LAST: the final pass also fetches each term's coefficient from the source
// and writes it in sorted order, so the segment sums read contiguous values.
// KONLY: index-packed keys (the term index in the bits below the digits) and
// no payload; the last pass then reads the term's phase / sign byte phs[idx],
// writes the coefficient with its sign folded and replaces the index bits of
// the key by the phase bit.
template <class Src, bool LAST, int ITEMS, bool KONLY>
__global__ void __launch_bounds__(kThreads, KONLY ? (ITEMS <= 12 ? 4 : 3)
                                                  : (ITEMS <= 8 ? 4 : (ITEMS <= 12 ? 3 : 2)))
    k_radix_pass(const u64* __restrict__ kin, const u32* __restrict__ vin, u64* __restrict__ kout,
                 u32* __restrict__ vout, u32 n, int shift, int bits,
                 const u32* __restrict__ bstart, u32* lb, u32* tile_ctr, int* status, Src src,
                 double* __restrict__ val_out, const uint2* __restrict__ phs, u64 imask,
                 u32 pf_ahead, u32* lb_next, int lbw) {
    extern __shared__ __align__(16) unsigned char dsm[];
    u64* skeys = reinterpret_cast<u64*>(dsm);
    u32* svals = reinterpret_cast<u32*>(dsm + sizeof(u64) * (kThreads * ITEMS));
    __shared__ RadixSmem S;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        const u32 t = atomicAdd(tile_ctr, 1u);
        S.tile = t;
        // The tile about one wave ahead goes to L2 now, so the CTA that takes
        // it finds its keys there instead of waiting on DRAM.
        const u32 pt = t + pf_ahead;
        if (pf_ahead && (u64)(pt + 1) * (kThreads * ITEMS) <= n) {
            prefetch_l2(kin + (size_t)pt * (kThreads * ITEMS), 8u * (kThreads * ITEMS));
            if constexpr (!KONLY)
                prefetch_l2(vin + (size_t)pt * (kThreads * ITEMS), 4u * (kThreads * ITEMS));
        }
    }
    for (int i = tid; i < kWarps * kRadix; i += kThreads) S.whist[i] = 0;
    __syncthreads();
    const u32 tile = S.tile;
    const u32 base = tile * (u32)(kThreads * ITEMS);
    const u32 dmask = (1u << bits) - 1u;
    // The next pass's look-back words (the other of two regions; the pass
    // before this one used it and is done): each tile clears its own, so no
    // pass needs a separate clearing launch.  kThreads == kRadix.
    if (lb_next) lb_next[(size_t)tile * kRadix + tid] = 0u;

    u64 keys[ITEMS];
    u32 vals[KONLY ? 1 : ITEMS];
    u32 rank[(ITEMS + 1) / 2];  // two 16-bit in-warp ranks per word (a warp ranks < 2^16 keys)
    const u32 wbase = base + (u32)warp * (ITEMS * 32);
#pragma unroll
    for (int t = 0; t < ITEMS; ++t) {
        const u32 idx = wbase + t * 32 + lane;
        keys[t] = idx < n ? kin[idx] : 0ull;
        if constexpr (!KONLY) vals[t] = idx < n ? vin[idx] : kSentinel;
    }
    u32* wh = S.whist + warp * kRadix;
#pragma unroll
    for (int t = 0; t < ITEMS; ++t) {
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
        const u32 r = before + __popc(peers & lanemask_lt());
        rank[t / 2] = (t & 1) ? (rank[t / 2] | (r << 16)) : r;
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
#pragma unroll
    for (int w = 0; w < kWarps; ++w) S.whist[w * kRadix + d] += bl;
    // the aggregate goes out first; the scatter into shared memory needs only
    // tile positions and runs while the predecessors' prefixes arrive
    lb_publish(lb + d, tile, kRadix, run);
    __syncthreads();
#pragma unroll
    for (int t = 0; t < ITEMS; ++t) {
        if (wbase + t * 32 + lane < n) {
            const u32 dd = (u32)(keys[t] >> shift) & dmask;
            const u32 pos = S.whist[warp * kRadix + dd] + ((rank[t / 2] >> ((t & 1) * 16)) & 0xffffu);
            skeys[pos] = keys[t];
            if constexpr (!KONLY) svals[pos] = vals[t];
        }
    }
    // look-back window (predecessors read per L2 round trip) in the low 8
    // bits of lbw, hot polls before backing off above them
    const int win = lbw & 0xff;
    const u32 hot = (u32)lbw >> 8;
    const u32 excl = win >= 16 ? lb_walk<16>(lb + d, tile, kRadix, run, status, hot)
                     : win >= 8 ? lb_walk<8>(lb + d, tile, kRadix, run, status, hot)
                     : win >= 4 ? lb_walk<4>(lb + d, tile, kRadix, run, status, hot)
                                : lb_walk<2>(lb + d, tile, kRadix, run, status, hot);
    S.gofs[d] = bstart[d] + excl - bl;  // modulo 2^32; gofs[d] + p >= 0 for p >= bl
    __syncthreads();
    const u32 tile_n = min((u32)(kThreads * ITEMS), n - base);
    if constexpr (KONLY && LAST) {
        // kGather terms per thread at a time: all their gathers (phase byte,
        // coefficient) are issued before the first one is used.
        constexpr int kGather = 8;
        for (u32 p0 = 0; p0 < tile_n; p0 += kGather * kThreads) {
            u64 kk[kGather];
            u32 gg[kGather], ph[kGather];
            double vv[kGather];
#pragma unroll
            for (int b = 0; b < kGather; ++b) {
                const u32 p = p0 + (u32)b * kThreads + tid;
                gg[b] = 0xffffffffu;
                kk[b] = 0;
                ph[b] = 0;
                vv[b] = 0.0;
                if (p < tile_n) {
                    const u64 k = skeys[p];
                    const u32 dd = (u32)(k >> shift) & dmask;
                    const u32 idx = (u32)(k & imask);
                    kk[b] = k;
                    gg[b] = S.gofs[dd] + p;
                    if (idx < n) {
                        src.flags_value(idx, phs, ph[b], vv[b]);
                    } else {
                        gg[b] = n;  // reported below
                    }
                }
            }
#pragma unroll
            for (int b = 0; b < kGather; ++b) {
                if (gg[b] < n) {
                    kout[gg[b]] = (kk[b] & ~imask) | (u64)(ph[b] & 1u);
                    val_out[gg[b]] = (ph[b] & 2u) ? -vv[b] : vv[b];
                } else if (gg[b] != 0xffffffffu) {
                    raise_status(status, PL_ERR_INTERNAL);
                }
            }
        }
        return;
    }
    if (tile_n == (u32)(kThreads * ITEMS) && (KONLY || !LAST)) {
        // full tile: half of a thread's keys and offsets at a time are loaded
        // before their stores
        constexpr int kH = ITEMS / 2;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            u64 kk[kH];
            u32 gg[kH];
#pragma unroll
            for (int t = 0; t < kH; ++t) kk[t] = skeys[tid + (h * kH + t) * kThreads];
#pragma unroll
            for (int t = 0; t < kH; ++t)
                gg[t] = S.gofs[(u32)(kk[t] >> shift) & dmask] + (u32)(tid + (h * kH + t) * kThreads);
#pragma unroll
            for (int t = 0; t < kH; ++t) {
                if (gg[t] >= n) {
                    raise_status(status, PL_ERR_INTERNAL);
                    continue;
                }
                kout[gg[t]] = kk[t];
                if constexpr (!KONLY) vout[gg[t]] = svals[tid + (h * kH + t) * kThreads];
            }
        }
        return;
    }
    for (u32 p = tid; p < tile_n; p += kThreads) {
        const u64 k = skeys[p];
        const u32 dd = (u32)(k >> shift) & dmask;
        const u32 g = S.gofs[dd] + p;
        if (g >= n) {
            raise_status(status, PL_ERR_INTERNAL);
        } else if constexpr (KONLY) {
            kout[g] = k;
        } else {
            const u32 pv = svals[p];
            kout[g] = k;
            vout[g] = pv;
            if (LAST) val_out[g] = src.value(pv & kIdxMask);
        }
    }
}

constexpr size_t radix_smem(int items) { return (sizeof(u64) + sizeof(u32)) * kThreads * items; }
constexpr size_t radix_smem_konly(int items) { return sizeof(u64) * kThreads * items; }

// ---------------------------------------------------------------------------
// 3b. Digit pass with 10-bit digits over index-packed keys (1024 buckets):
//     a product's 40 varying x / z bits sort in 4 passes instead of 5.  The
//     same onesweep structure as k_radix_pass; each thread owns 4
//     consecutive buckets (scan, look-back, offsets), the per-warp counts
//     are 16-bit, and the four look-back walks run interleaved (all their
//     window loads in flight at once).
// ---------------------------------------------------------------------------
constexpr int kRadixW = 1024;
constexpr int kBpt = kRadixW / kThreads;  // buckets per thread

struct RadixSmemW {
    u16 whist[kWarps * kRadixW];  // per warp: digit counts, then tile positions
    u32 gofs[kRadixW];
    u32 swarp[kWarps];
    u32 tile;
};

// Decoupled look-back for this thread's kBpt buckets (columns col, col + 1,
// ...) at once; publishes each inclusive prefix and returns the exclusive
// ones in excl.  Bounded like lb_walk.
template <int W>
__device__ __forceinline__ void lb_walk_w(u32* lb, u32 tile, u32 col, const u32 (&cnt)[kBpt],
                                          u32 (&excl)[kBpt], int* status) {
#pragma unroll
    for (int b = 0; b < kBpt; ++b) excl[b] = 0;
    if (tile == 0) return;
    i64 t[kBpt];
    bool done[kBpt];
#pragma unroll
    for (int b = 0; b < kBpt; ++b) {
        t[b] = (i64)tile - 1;
        done[b] = false;
    }
    u32 spins = 0;
    for (;;) {
        u32 w[kBpt][W];
#pragma unroll
        for (int b = 0; b < kBpt; ++b)
#pragma unroll
            for (int k = 0; k < W; ++k)
                w[b][k] = (!done[b] && t[b] - k >= 0)
                              ? ld_volatile(lb + (size_t)(t[b] - k) * kRadixW + col + b)
                              : kFlagPre;
        bool all = true, moved = false;
#pragma unroll
        for (int b = 0; b < kBpt; ++b) {
            if (done[b]) continue;
            int k = 0;
            for (; k < W; ++k) {
                const u32 fl = w[b][k] >> 30;
                if (fl == 0) break;
                excl[b] += w[b][k] & kCountMask;
                if (fl == 2) {
                    done[b] = true;
                    break;
                }
            }
            if (!done[b]) {
                t[b] -= k;
                all = false;
                moved = moved || k > 0;
            } else {
                moved = true;
            }
        }
        if (all) break;
        if (!moved) {
            if (++spins > g_spin_limit) {
                raise_status(status, PL_ERR_TIMEOUT);
                break;
            }
            if (spins > 64) __nanosleep(64);
        }
    }
#pragma unroll
    for (int b = 0; b < kBpt; ++b)
        st_volatile(lb + (size_t)tile * kRadixW + col + b, kFlagPre | ((excl[b] + cnt[b]) & kCountMask));
}

template <class Src, bool LAST, int ITEMS>
__global__ void __launch_bounds__(kThreads, ITEMS <= 12 ? 4 : 3)
    k_radix_pass_w(const u64* __restrict__ kin, u64* __restrict__ kout, u32 n, int shift,
                   int bits, const u32* __restrict__ bstart, u32* lb, u32* tile_ctr, int* status,
                   Src src, double* __restrict__ val_out, const uint2* __restrict__ phs,
                   u64 imask, u32 pf_ahead, u32* lb_next, int lbw) {
    constexpr u32 kTile = (u32)(kThreads * ITEMS);
    extern __shared__ __align__(16) unsigned char dsm[];
    u64* skeys = reinterpret_cast<u64*>(dsm);
    __shared__ __align__(16) RadixSmemW S;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        const u32 t = atomicAdd(tile_ctr, 1u);
        S.tile = t;
        const u32 pt = t + pf_ahead;
        if (pf_ahead && (u64)(pt + 1) * kTile <= n)
            prefetch_l2(kin + (size_t)pt * kTile, 8u * kTile);
    }
    // 16 KB of 16-bit counts: four 16-byte stores per thread
#pragma unroll
    for (int i = 0; i < 4; ++i)
        reinterpret_cast<uint4*>(S.whist)[tid + i * kThreads] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    const u32 tile = S.tile;
    const u32 base = tile * kTile;
    const u32 dmask = (1u << bits) - 1u;
    const u32 col = (u32)tid * kBpt;  // this thread's first bucket
    if (lb_next) {
#pragma unroll
        for (int b = 0; b < kBpt; ++b) lb_next[(size_t)tile * kRadixW + col + b] = 0u;
    }
    u64 keys[ITEMS];
    u32 rank[(ITEMS + 1) / 2];
    const u32 wbase = base + (u32)warp * (ITEMS * 32);
#pragma unroll
    for (int t = 0; t < ITEMS; ++t) {
        const u32 idx = wbase + t * 32 + lane;
        keys[t] = idx < n ? kin[idx] : 0ull;
    }
    u16* wh = S.whist + warp * kRadixW;
#pragma unroll
    for (int t = 0; t < ITEMS; ++t) {
        const bool valid = (wbase + t * 32 + lane) < n;
        const u32 d = valid ? ((u32)(keys[t] >> shift) & dmask) : kSentinel;
        const u32 peers = __match_any_sync(0xffffffffu, d);
        const int leader = __ffs(peers) - 1;
        u32 before = 0;
        if (valid && lane == leader) {
            before = wh[d];
            wh[d] = (u16)(before + __popc(peers));
        }
        before = __shfl_sync(0xffffffffu, before, leader);
        const u32 r = before + __popc(peers & lanemask_lt());
        rank[t / 2] = (t & 1) ? (rank[t / 2] | (r << 16)) : r;
        __syncwarp();
    }
    __syncthreads();
    // per bucket: exclusive prefix over warps; the thread's 4 buckets in a row
    u32 run[kBpt], tot = 0;
#pragma unroll
    for (int b = 0; b < kBpt; ++b) {
        u32 r = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const u32 c = S.whist[w * kRadixW + col + b];
            S.whist[w * kRadixW + col + b] = (u16)r;
            r += c;
        }
        run[b] = r;
        tot += r;
    }
    u32 total;
    u32 bl[kBpt];
    bl[0] = block_excl_scan(tot, S.swarp, total);
#pragma unroll
    for (int b = 1; b < kBpt; ++b) bl[b] = bl[b - 1] + run[b - 1];
#pragma unroll
    for (int b = 0; b < kBpt; ++b) {
#pragma unroll
        for (int w = 0; w < kWarps; ++w) S.whist[w * kRadixW + col + b] += (u16)bl[b];
        lb_publish(lb + col + b, tile, kRadixW, run[b]);
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < ITEMS; ++t) {
        if (wbase + t * 32 + lane < n) {
            const u32 dd = (u32)(keys[t] >> shift) & dmask;
            const u32 pos = (u32)S.whist[warp * kRadixW + dd] +
                            ((rank[t / 2] >> ((t & 1) * 16)) & 0xffffu);
            skeys[pos] = keys[t];
        }
    }
    u32 excl[kBpt];
    if ((lbw & 0xff) >= 8) lb_walk_w<8>(lb, tile, col, run, excl, status);
    else if ((lbw & 0xff) >= 4) lb_walk_w<4>(lb, tile, col, run, excl, status);
    else lb_walk_w<2>(lb, tile, col, run, excl, status);
#pragma unroll
    for (int b = 0; b < kBpt; ++b) S.gofs[col + b] = bstart[col + b] + excl[b] - bl[b];
    __syncthreads();
    const u32 tile_n = min(kTile, n - base);
    if constexpr (LAST) {
        constexpr int kGather = 8;
        for (u32 p0 = 0; p0 < tile_n; p0 += kGather * kThreads) {
            u64 kk[kGather];
            u32 gg[kGather], ph[kGather];
            double vv[kGather];
#pragma unroll
            for (int q = 0; q < kGather; ++q) {
                const u32 p = p0 + (u32)q * kThreads + tid;
                gg[q] = 0xffffffffu;
                kk[q] = 0;
                ph[q] = 0;
                vv[q] = 0.0;
                if (p < tile_n) {
                    const u64 k = skeys[p];
                    const u32 idx = (u32)(k & imask);
                    kk[q] = k;
                    gg[q] = S.gofs[(u32)(k >> shift) & dmask] + p;
                    if (idx < n) src.flags_value(idx, phs, ph[q], vv[q]);
                    else gg[q] = n;  // reported below
                }
            }
#pragma unroll
            for (int q = 0; q < kGather; ++q) {
                if (gg[q] < n) {
                    kout[gg[q]] = (kk[q] & ~imask) | (u64)(ph[q] & 1u);
                    val_out[gg[q]] = (ph[q] & 2u) ? -vv[q] : vv[q];
                } else if (gg[q] != 0xffffffffu) {
                    raise_status(status, PL_ERR_INTERNAL);
                }
            }
        }
        return;
    }
    for (u32 p = tid; p < tile_n; p += kThreads) {
        const u64 k = skeys[p];
        const u32 g = S.gofs[(u32)(k >> shift) & dmask] + p;
        if (g >= n) raise_status(status, PL_ERR_INTERNAL);
        else kout[g] = k;
    }
}




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

// Keep-filter applied when a segment is closed.  With on = 1 the zero and
// cutoff filters are decided here and every warp adds its survivors to the
// count of its kETile-term tile, so the emit pass needs no look-back; with
// on = 0 (a weight filter, which needs the unpacked key) every head is
// marked kept and the emit pass filters.
struct FoldFilter {
    int on;
    double cutoff;
    u32* tile_kept;
    double2* seg2;   // kCanonSplit: (phase-0 sum, phase-1 sum) of each head's record
    double2* rpre;   // per fold range: the sums of its terms before its first head
    double2* ptail;  // per pending segment: its sums at the end of its range
    // kCanonSplit head records: the heads of fold range g sit at slots
    // [g * kFoldSpan, g * kFoldSpan + rng_heads[g]) in key order -- the sorted
    // key in rkey, the two sums in seg2 -- and rng_kept[g] counts the output
    // terms they give.
    u64* rkey;
    u32* rng_heads;
    u32* rng_kept;
};

// canonicalize() on index-packed keys: the sort key is (x, z) only and the
// phase bit sits in bit 0 of the sorted key; every (x, z) segment keeps two
// sums, phase 0 and phase 1, each over its members in index order -- the
// sums a stable sort by (x, z, phase) followed by left-to-right folding
// gives.  Each can become one output term.  Values arrive with the sign
// folded in.
constexpr int kCanonSplit = 3;

// Segment fold.  A warp owns 1024 consecutive sorted terms, staged in shared
// memory; lane L folds its own 32 terms left to right (32 independent
// chains per warp), the reference's order (PauliSumOperations.h:443-455).
// Segments that cross lane borders: a lane with a head knows the segment
// open at the end of its span; the lane after it continues that segment
// over its span term by term; longer chains of headless lanes combine the
// lanes' partial sums in a fixed tree, and the lane that closes the segment
// folds its own terms onto the result term by term.  Every segment within
// three lanes is therefore summed exactly in the reference's order, and
// every other one in a fixed order (deterministic; within 1e-12 of the
// summed magnitudes).  The warp that holds a segment's head owns it; one
// still open at the end of the range continues over the staged lookahead
// (term by term) and otherwise goes to the carry pass (k_fold_carry), which
// adds the following ranges' prefix partials.
// segflag[head] = 1 kept, 3 dropped, 2 pending; non-heads get 0.
// wfirst[warp] = offset of the range's first head, kNoHead if none.
constexpr int kFoldWarps = 4;
constexpr int kLaneSpan = 32;
constexpr u32 kFoldSpan = 32u * kLaneSpan;  // 1024 terms per warp
constexpr u32 kLook = 64;                   // terms after the range staged as well
constexpr u32 kLookSlot = 33u * 32u;        // lane spans padded to 33 slots (no bank conflicts)
constexpr u32 kFoldSlots = kLookSlot + kLook;
constexpr u32 kFoldChunks = 32u + kLook / 32u;
// per warp: the staged values, then per 32-term chunk a word of head bits and
// a word of sign bits (chunk c < 32 is lane c's span)
constexpr size_t kFoldWarpSmem = kFoldSlots * 8 + kFoldChunks * 8;
constexpr size_t kFoldSmem = ((kFoldWarpSmem + 15) & ~size_t(15)) * kFoldWarps;
constexpr u32 kNoHead = 0xffffffffu;
constexpr int kEItems = 8;
constexpr u32 kETile = kThreads * kEItems;  // 2048 terms per emit tile

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

// One term onto a running sum: kCanon folds the sign into the value, kProp
// keeps the sign-0 and sign-1 sums apart (S0 - S1 at the close), kCanonSplit
// the phase-0 and phase-1 sums (bit 31 of p is the phase there).
template <int MODE>
__device__ __forceinline__ void fold_add(double& r0, double& r1, double v, u32 p) {
    const bool neg = (p >> 31) != 0;
    if (MODE == kCanonSplit) {  // branch-free, as fold_term below
        r0 = dadd(r0, neg ? 0.0 : v);
        r1 = dadd(r1, neg ? v : 0.0);
    } else if (MODE == kCanon) r0 = dadd(r0, neg ? -v : v);
    else if (MODE == kCombine) r0 = dadd(r0, v);
    else if (neg) r1 = dadd(r1, v);
    else r0 = dadd(r0, v);
}

// The same for a staged term whose kCanon value already carries its sign.
//
// kCanonSplit adds every term to both sums, +0.0 to the one it does not
// belong to: a sum that starts at +0.0 never becomes -0.0, so adding +0.0
// leaves it unchanged and the result is bit-identical to the branch.
template <int MODE>
__device__ __forceinline__ void fold_term(double& r0, double& r1, double v, u32 neg) {
    if (MODE == kCanonSplit) {
        r0 = dadd(r0, neg ? 0.0 : v);
        r1 = dadd(r1, neg ? v : 0.0);
    } else if (MODE == kProp && neg) {
        r1 = dadd(r1, v);
    } else {
        r0 = dadd(r0, v);
    }
}

// Bit 31 of a term's fold word: the sign (kCanon, kProp) from the payload,
// or the phase (kCanonSplit) from bit 0 of the sorted key.
template <int MODE>
__device__ __forceinline__ u32 fold_word(const SegCtx& C, u32 e, u64 key) {
    if (MODE == kCanonSplit) return ((u32)key & 1u) << 31;
    return C.pay[e];
}

// One of a kCanonSplit head's two sums gives an output term: zero and cutoff
// filters of canonicalize() + cutoff().
__device__ __forceinline__ u32 split_kept(double r, double cutoff) {
    return (r != 0.0 && (cutoff <= 0.0 || fabs(r) >= cutoff)) ? 1u : 0u;
}

template <int MODE>
__device__ __forceinline__ u32 fold_close(double* segval, u8* segflag, i64 h, double r0,
                                          double r1, const FoldFilter& F) {
    if (MODE == kCanonSplit) {
        // h is the head's record slot; the emit re-applies the same filters
        F.seg2[h] = make_double2(r0, r1);
        return split_kept(r0, F.cutoff) + split_kept(r1, F.cutoff);
    }
    const double v = MODE == kProp ? dadd(r0, -r1) : r0;
    segval[h] = v;
    bool keep = true;
    if (F.on) {
        keep = (MODE == kCombine) || (v != 0.0);
        if (F.cutoff > 0.0) keep = keep && (fabs(v) >= F.cutoff);
    }
    segflag[h] = keep ? 1 : 3;
    return keep ? 1u : 0u;
}

// Where the fold takes each sorted term's fold word and coefficient: from
// the sorted arrays (NoGather), or -- for a product whose last digit pass
// moved keys only, index bits kept -- from the term's index: its phase / sign
// bits from the bit planes and its coefficient lhs_j * rhs_i from the
// operands (ProdGather), the values the last pass would have written.
struct NoGather {
    static constexpr bool kOn = false;
    __device__ __forceinline__ void get(u64, u32&, double&) const {}
};
template <int AS>
struct ProdGather {
    ProdSrc<AS> src;
    const uint2* phs;
    u64 imask;
    u32 n;  // products
    int* status;
    static constexpr bool kOn = true;
    __device__ __forceinline__ void get(u64 key, u32& pe, double& ve) const {
        const u32 idx = (u32)(key & imask);
        u32 fl = 0;
        double v = 0.0;
        if (idx < n) src.flags_value(idx, phs, fl, v);
        else raise_status(status, PL_ERR_INTERNAL);
        pe = (fl & 1u) << 31;
        ve = (fl & 2u) ? -v : v;
    }
};

template <int MODE, class G = NoGather>
__global__ void __launch_bounds__(32 * kFoldWarps, 6)
    k_fold(SegCtx C, double* segval, u8* segflag, u32* wfirst, u32* long_list, u32* counters,
           FoldFilter F, G g) {
    extern __shared__ __align__(16) unsigned char fsm[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const u32 gwarp = blockIdx.x * kFoldWarps + warp;
    const u32 w0 = gwarp * kFoldSpan;
    if (w0 >= C.n) return;
    const u32 w1 = min(w0 + kFoldSpan, C.n);
    const u32 cnt = w1 - w0;
    if (lane == 0 && (C.n - w0) >= kFoldSpan + kLook) {
        // the whole range and its lookahead go to L2 at once, so the staging
        // batches after the first find them there instead of each waiting on
        // DRAM in turn
        prefetch_l2(C.keys + w0, 8u * (kFoldSpan + kLook));
        if (!G::kOn) prefetch_l2(C.vals + w0, 8u * (kFoldSpan + kLook));
        if (MODE != kCanonSplit && C.pay) prefetch_l2(C.pay + w0, 4u * (kFoldSpan + kLook));
    }
    unsigned char* base = fsm + ((kFoldWarpSmem + 15) & ~size_t(15)) * warp;
    double* sv = reinterpret_cast<double*>(base);
    u32* hbw = reinterpret_cast<u32*>(base + 8 * kFoldSlots);
    u32* nbw = hbw + kFoldChunks;
    // ---- staging: coalesced loads, head flags, non-head segflag = 0
    u64 ck = 0;
    u32 cp = 0;
    if (w0 > 0) {
        ck = C.keys[w0 - 1];
        cp = fold_word<MODE>(C, w0 - 1, ck);
    }
    u32 first = kNoHead;
    u32 nhead = 0;  // kCanonSplit: heads of the range so far (their record slots)
    // kBatch chunks of loads in flight per lane, then the head flags of those
    // chunks; per chunk, a word of head bits and a word of sign bits
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
            if constexpr (!G::kOn) {
                pe[b] = valid ? fold_word<MODE>(C, w0 + i, ke[b]) : 0u;
                ve[b] = valid ? C.vals[w0 + i] : 0.0;
            }
        }
        if constexpr (G::kOn) {
            // all the batch's keys are in flight first; then their gathers
#pragma unroll
            for (int b = 0; b < kBatch; ++b) {
                pe[b] = 0u;
                ve[b] = 0.0;
                if ((c0 + b) * 32 + lane < cnt) g.get(ke[b], pe[b], ve[b]);
            }
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
            bool head = false, neg = false;
            if (i < cnt) {
                head = (e == 0) || !lane_same_key(C, e, ke[b], kp, pe[b], pp);
                neg = (pe[b] >> 31) != 0;
                sv[c * 33 + lane] = (MODE == kCanon && neg) ? -ve[b] : ve[b];
                if (MODE != kCanonSplit && !head) segflag[e] = 0;
            }
            const u32 hb = __ballot_sync(0xffffffffu, head);
            const u32 nb = __ballot_sync(0xffffffffu, neg);
            if (MODE == kCanonSplit) {
                if (head) F.rkey[w0 + nhead + __popc(hb & lanemask_lt())] = ke[b];
                nhead += __popc(hb);
            }
            if (lane == 0 && c < 32) {
                hbw[c] = hb;
                nbw[c] = nb;
            }
            if (first == kNoHead && hb) first = c * 32 + (u32)(__ffs(hb) - 1);
            ck = __shfl_sync(0xffffffffu, ke[b], 31);
            cp = __shfl_sync(0xffffffffu, pe[b], 31);
        }
    }
    // Up to kLook terms after the range, for the continuation of a segment
    // still open at its end (their segflag belongs to the next range); lanes
    // past the lookahead count as heads, which stops the continuation there.
    const u32 look = w1 < C.n ? min(kLook, C.n - w1) : 0u;
    if (look) {
        u64 ke[kLook / 32];
        u32 pe[kLook / 32];
        double ve[kLook / 32];
#pragma unroll
        for (int b = 0; b < (int)(kLook / 32); ++b) {
            const u32 q = (u32)b * 32 + lane;
            const bool valid = q < look;
            ke[b] = valid ? C.keys[w1 + q] : 0ull;
            if constexpr (G::kOn) {
                pe[b] = 0u;
                ve[b] = 0.0;
                if (valid) g.get(ke[b], pe[b], ve[b]);
            } else {
                pe[b] = valid ? fold_word<MODE>(C, w1 + q, ke[b]) : 0u;
                ve[b] = valid ? C.vals[w1 + q] : 0.0;
            }
        }
#pragma unroll
        for (int b = 0; b < (int)(kLook / 32); ++b) {
            const u32 q = (u32)b * 32 + lane;
            u64 kp = __shfl_up_sync(0xffffffffu, ke[b], 1);
            u32 pp = __shfl_up_sync(0xffffffffu, pe[b], 1);
            if (lane == 0) {
                kp = ck;
                pp = cp;
            }
            bool head = true, neg = false;
            if (q < look) {
                head = !lane_same_key(C, w1 + q, ke[b], kp, pe[b], pp);
                neg = (pe[b] >> 31) != 0;
                sv[kLookSlot + q] = (MODE == kCanon && neg) ? -ve[b] : ve[b];
            }
            const u32 hb = __ballot_sync(0xffffffffu, head);
            const u32 nb = __ballot_sync(0xffffffffu, neg);
            if (lane == 0) {
                hbw[32 + b] = hb;
                nbw[32 + b] = nb;
            }
            ck = __shfl_sync(0xffffffffu, ke[b], 31);
            cp = __shfl_sync(0xffffffffu, pe[b], 31);
        }
    }
    if (lane == 0) wfirst[gwarp] = first;
    __syncwarp();
    // ---- phase 1: each lane folds the segments that start inside its span,
    // and the terms before its first head (its whole span when it has none)
    // from zero: its prefix partial
    const u32 a = (u32)lane * kLaneSpan;
    const u32 sa = (u32)lane * 33u;
    const u32 lcnt = cnt > a ? min(cnt - a, (u32)kLaneSpan) : 0u;
    const u32 HB = lcnt ? hbw[lane] : 0u;  // head / sign bits of the lane's span
    const u32 NB = lcnt ? nbw[lane] : 0u;
    u32 fh = lcnt;  // prefix length (terms before the lane's first head)
    i64 h = -1;
    double r0 = 0.0, r1 = 0.0, p0 = 0.0, p1 = 0.0;
    u32 kept = 0;
    // kCanonSplit closes a head by its record slot: w0 + (heads of the range
    // before it), i.e. the heads of the earlier lanes' spans plus the lane's
    // own earlier heads
    i64 hs = -1;
    u32 nslot = 0;
    if (MODE == kCanonSplit) {
        const u32 c = (u32)__popc(HB);
        u32 inc = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += t;
        }
        nslot = w0 + inc - c;
    }
    for (u32 i = 0; i < lcnt; ++i) {
        const double v = sv[sa + i];
        if ((HB >> i) & 1u) {
            if (h >= 0) kept += fold_close<MODE>(segval, segflag, MODE == kCanonSplit ? hs : h, r0, r1, F);
            else fh = i;
            h = (i64)(w0 + a + i);
            hs = (i64)(nslot++);
            r0 = 0.0;
            r1 = 0.0;
        }
        if (h >= 0) fold_term<MODE>(r0, r1, v, (NB >> i) & 1u);
        else fold_term<MODE>(p0, p1, v, (NB >> i) & 1u);
    }
    // ---- phase 2: the segment open at the end of each lane's span, (oh, o0,
    // o1) with oh = -1 for one that began before the range.  A lane with a
    // head knows it.  A headless lane right after a lane with a head folds its
    // span onto that segment term by term (the reference's order); every
    // longer chain of headless lanes adds the lanes' prefix partials in a
    // fixed tree (segmented scan over the lanes), so results are
    // deterministic and equal the reference's order for every segment that
    // spans at most three lanes.
    const bool hh = fh < lcnt;
    // kCanonSplit: oh travels as the head's record slot
    i64 oh = hh ? (MODE == kCanonSplit ? hs : h) : -1;
    double o0 = hh ? r0 : p0, o1 = hh ? r1 : p1;
    bool known = hh;
    {
        const i64 ph = __shfl_up_sync(0xffffffffu, oh, 1);
        const double q0 = __shfl_up_sync(0xffffffffu, o0, 1);
        const double q1 = __shfl_up_sync(0xffffffffu, o1, 1);
        const int pk = __shfl_up_sync(0xffffffffu, (int)hh, 1);
        if (lane > 0 && !hh && pk) {
            oh = ph;
            o0 = q0;
            o1 = q1;
            for (u32 i = 0; i < lcnt; ++i) fold_term<MODE>(o0, o1, sv[sa + i], (NB >> i) & 1u);
            known = true;
        }
    }
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const i64 ph = __shfl_up_sync(0xffffffffu, oh, d);
        const double q0 = __shfl_up_sync(0xffffffffu, o0, d);
        const double q1 = __shfl_up_sync(0xffffffffu, o1, d);
        const int pk = __shfl_up_sync(0xffffffffu, (int)known, d);
        if (lane >= d && !known) {
            oh = ph;
            o0 = dadd(q0, o0);
            o1 = dadd(q1, o1);
            known = pk != 0;
        }
    }
    // ---- close: a lane with a head folds the terms before it onto the
    // segment coming in from the left (term by term); the warp's first head
    // gets the range's prefix partial instead (the terms of a segment that
    // began in an earlier range), which the carry pass adds to it.
    double rp0 = 0.0, rp1 = 0.0;
    {
        i64 cin = __shfl_up_sync(0xffffffffu, oh, 1);
        double q0 = __shfl_up_sync(0xffffffffu, o0, 1);
        double q1 = __shfl_up_sync(0xffffffffu, o1, 1);
        if (lane == 0) {
            cin = -1;
            q0 = 0.0;
            q1 = 0.0;
        }
        if (hh) {
            for (u32 i = 0; i < fh; ++i) fold_term<MODE>(q0, q1, sv[sa + i], (NB >> i) & 1u);
            if (cin >= 0) {
                kept += fold_close<MODE>(segval, segflag, cin, q0, q1, F);
            } else {
                rp0 = q0;
                rp1 = q1;
            }
        }
    }
    const i64 ch = __shfl_sync(0xffffffffu, oh, 31);
    const double c0 = __shfl_sync(0xffffffffu, o0, 31);
    const double c1 = __shfl_sync(0xffffffffu, o1, 31);
    {
        // the range's prefix partial, for the carry pass of an earlier range
        const u32 fl = first == kNoHead ? 31u : first / kLaneSpan;
        const double e0 = __shfl_sync(0xffffffffu, first == kNoHead ? o0 : rp0, (int)fl);
        const double e1 = __shfl_sync(0xffffffffu, first == kNoHead ? o1 : rp1, (int)fl);
        if (lane == 0) F.rpre[gwarp] = make_double2(e0, e1);
    }
    // ---- the open segment at the end of the range, when this warp owns it:
    // the staged lookahead continues it term by term; one still open after
    // it goes to the carry pass with its value before the lookahead.
    if (ch >= 0 && lane == 0) {
        if (w1 == C.n) {
            kept += fold_close<MODE>(segval, segflag, ch, c0, c1, F);
        } else {
            double d0 = c0, d1 = c1;
            bool closed = false;
            for (u32 q = 0; q < look; ++q) {
                const u32 wq = 32u + (q >> 5), bq = q & 31u;
                if ((hbw[wq] >> bq) & 1u) {
                    closed = true;
                    break;
                }
                fold_term<MODE>(d0, d1, sv[kLookSlot + q], (nbw[wq] >> bq) & 1u);
            }
            if (closed || w1 + look == C.n) {
                kept += fold_close<MODE>(segval, segflag, ch, d0, d1, F);
            } else {
                if (MODE != kCanonSplit) segflag[ch] = 2;
                const u32 k = atomicAdd(&counters[2], 1u);
                long_list[k] = (u32)ch;
                F.ptail[k] = make_double2(c0, c1);
            }
        }
    }
    if (F.on) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) kept += __shfl_xor_sync(0xffffffffu, kept, o);
        if (MODE == kCanonSplit) {
            if (lane == 0) {
                F.rng_heads[gwarp] = nhead;
                F.rng_kept[gwarp] = kept;
            }
        } else if (lane == 0 && kept) {
            atomicAdd(&F.tile_kept[w0 / kETile], kept);
        }
    }
}

// Carry pass: a segment still open after its range and the lookahead (the
// pending list, counters[2]) continues through the following ranges up to
// the first one with a head; its sum is its value at the end of its range
// plus those ranges' prefix partials, added 32 ranges at a time in a fixed
// tree.  One warp per pending segment.
//
// SCAN (kCanonSplit, 1024-thread blocks): the last block to finish then turns
// the ranges' kept counts into their output offsets (the tile scan), so the
// record emit follows without a launch in between.  done: a zeroed counter.
__device__ __forceinline__ void tile_scan_block(const u32* tile_kept, u32 tiles, u32* tile_off,
                                                i64* d_out_count, u32* sw);

template <int MODE, bool SCAN = false>
__global__ void __launch_bounds__(SCAN ? 1024 : 256)
    k_fold_carry(const u32* wfirst, u32 ngw, const u32* long_list, const u32* counters,
                 double* segval, u8* segflag, FoldFilter F, u32* rng_off = nullptr,
                 i64* d_out_count = nullptr, u32* done = nullptr) {
    const u32 npend = counters[2];
    const int lane = threadIdx.x & 31;
    const u32 nw = (gridDim.x * blockDim.x) >> 5;
    for (u32 li = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; li < npend; li += nw) {
        const u32 h = long_list[li];
        const double2 t = F.ptail[li];
        double a0 = t.x, a1 = t.y;
        for (u32 g0 = h / kFoldSpan + 1;; g0 += 32u) {
            const u32 g = g0 + (u32)lane;
            const bool end = g >= ngw || wfirst[g] != kNoHead;
            const u32 bal = __ballot_sync(0xffffffffu, end);
            const u32 last = bal ? (u32)(__ffs(bal) - 1) : 31u;
            double2 pr = make_double2(0.0, 0.0);
            if ((u32)lane <= last && g < ngw) pr = F.rpre[g];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                pr.x = dadd(pr.x, __shfl_xor_sync(0xffffffffu, pr.x, o));
                pr.y = dadd(pr.y, __shfl_xor_sync(0xffffffffu, pr.y, o));
            }
            a0 = dadd(a0, pr.x);
            a1 = dadd(a1, pr.y);
            if (bal) break;
        }
        if (lane == 0) {
            const u32 keep = fold_close<MODE>(segval, segflag, h, a0, a1, F);
            if (MODE == kCanonSplit) {
                if (keep) atomicAdd(&F.rng_kept[h / kFoldSpan], keep);  // h: a record slot
            } else if (F.on && keep) {
                atomicAdd(&F.tile_kept[h / kETile], keep);
            }
        }
    }
    if constexpr (SCAN) {
        __shared__ u32 s_last;
        __shared__ u32 sw[65];
        __syncthreads();  // this block's carries (and their count atomics) are done
        if (threadIdx.x == 0) {
            __threadfence();
            s_last = atomicAdd(done, 1u) == gridDim.x - 1 ? 1u : 0u;
        }
        __syncthreads();
        if (s_last) {
            __threadfence();
            tile_scan_block(F.rng_kept, ngw, rng_off, d_out_count, sw);
        }
    }
}

// Block-wide exclusive scan of one value per thread (NW warps).
template <int NW>
__device__ __forceinline__ u32 block_scan_n(u32 v, u32* s_warp, u32& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u32 inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const u32 t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const u32 c = lane < NW ? s_warp[lane] : 0u;
        u32 ci = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 t = __shfl_up_sync(0xffffffffu, ci, o);
            if (lane >= o) ci += t;
        }
        if (lane < NW) s_warp[32 + lane] = ci - c;
        if (lane == 31) s_warp[64] = ci;
    }
    __syncthreads();
    total = s_warp[64];
    const u32 r = s_warp[32 + warp] + inc - v;
    __syncthreads();
    return r;
}

// Output offsets of the emit tiles (exclusive scan of the kept counts; one
// CTA) and the output size.
// Up to 16 counts per thread (16384 tiles) are loaded at once, before any
// is added, so the scan waits for one round of loads instead of a chain.
__global__ void __launch_bounds__(1024) k_tile_scan(const u32* tile_kept, u32 tiles,
                                                    u32* tile_off, i64* d_out_count) {
    __shared__ u32 sw[65];
    tile_scan_block(tile_kept, tiles, tile_off, d_out_count, sw);
}

// The scan itself, by one 1024-thread block (counts read past L1: another
// block of the same kernel may have just added to them).
__device__ __forceinline__ void tile_scan_block(const u32* tile_kept, u32 tiles, u32* tile_off,
                                                i64* d_out_count, u32* sw) {
    const u32 per = (tiles + 1023u) / 1024u;
    const u32 b = threadIdx.x * per, e = min(b + per, tiles);
    u32 total;
    if (per <= 16) {
        u32 c[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) c[k] = b + k < e ? __ldcg(tile_kept + b + k) : 0u;
        u32 s = 0;
#pragma unroll
        for (int k = 0; k < 16; ++k) s += c[k];
        u32 run = block_scan_n<32>(s, sw, total);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            if (b + k < e) tile_off[b + k] = run;
            run += c[k];
        }
    } else {
        u32 s = 0;
        for (u32 i = b; i < e; ++i) s += __ldcg(tile_kept + i);
        u32 run = block_scan_n<32>(s, sw, total);
        for (u32 i = b; i < e; ++i) {
            tile_off[i] = run;
            run += __ldcg(tile_kept + i);
        }
    }
    if (threadIdx.x == 0) *d_out_count = (i64)total;
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
// 5. Emit: order-preserving compaction of the kept heads into the output.
// ---------------------------------------------------------------------------
template <int AS, class Src>
__device__ __forceinline__ void emit_key(const Src& src, const KeyLayout& L, u64 packed,
                                         const u32* pay, u32 pos, int mode, u64* xw, u64* zw,
                                         u32& fl) {
    if (L.nchunks == 1 && !Src::kVirtualKey) {
        u32 fv;
        unpack_key<AS>(L, packed, xw, zw, fv);
        fl = out_flags(fv, mode);
    } else {
        src.orig_key(pay[pos] & kIdxMask, xw, zw, fl);
        fl = mode == kCombine ? (fl & 3u) : (fl & 1u);
    }
}

template <int AS, class Src>
__device__ __forceinline__ void emit_term(const Src& src, const KeyLayout& L, u64 packed,
                                          const u32* pay, u32 e, int mode, double v, i64 o,
                                          const SoAOut& out, int* status) {
    if (o >= out.capacity) {
        raise_status(status, PL_ERR_CAPACITY);
        return;
    }
    u64 xw[AS], zw[AS];
    u32 f;
    emit_key<AS>(src, L, packed, pay, e, mode, xw, zw, f);
#pragma unroll
    for (int k = 0; k < AS; ++k) {
        out.x[(i64)k * out.capacity + o] = xw[k];
        out.z[(i64)k * out.capacity + o] = zw[k];
    }
    out.f[o] = (u8)f;
    out.v[o] = v;
}

// kCanonSplit emit from the fold's head records: one warp per fold range
// copies its kept terms -- a head's phase-0 term, then its phase-1 term (the
// canonical order: phase is the last key field) -- to the offset
// k_tile_scan gave the range.  The records are dense, so a range reads
// 24 bytes per head and nothing per non-head term.
constexpr int kRecBatch = 4;  // 32-head chunks whose loads are in flight at once
template <int AS>
__global__ void __launch_bounds__(kThreads)
    k_emit_records(KeyLayout L, const u64* __restrict__ rkey, const double2* __restrict__ rs,
                   const u32* __restrict__ rng_heads, const u32* __restrict__ rng_off, u32 ngw,
                   double cutoff, SoAOut out, int* status) {
    const int lane = threadIdx.x & 31;
    const u32 g = blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (g >= ngw) return;
    const u32 nh = rng_heads[g];
    const u32 w0 = g * kFoldSpan;
    i64 o = rng_off[g];
    if (lane == 0 && nh > 32 * kRecBatch) {
        // the range's later record batches go to L2 now (whole 16-byte units)
        prefetch_l2(rkey + w0, 8u * (nh & ~1u));
        prefetch_l2(rs + w0, 16u * nh);
    }
    for (u32 k0 = 0; k0 < nh; k0 += 32 * kRecBatch) {
        u64 key[kRecBatch];
        double2 v[kRecBatch];
#pragma unroll
        for (int b = 0; b < kRecBatch; ++b) {
            const u32 k = k0 + (u32)b * 32 + lane;
            key[b] = k < nh ? rkey[w0 + k] : 0ull;
            v[b] = k < nh ? rs[w0 + k] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int b = 0; b < kRecBatch; ++b) {
            const u32 k0b = split_kept(v[b].x, cutoff), k1b = split_kept(v[b].y, cutoff);
            const u32 c = k0b + k1b;
            u32 inc = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const u32 t = __shfl_up_sync(0xffffffffu, inc, d);
                if (lane >= d) inc += t;
            }
            const u32 tot = __shfl_sync(0xffffffffu, inc, 31);
            if (c) {
                u64 xw[AS], zw[AS];
                u32 fv;
                unpack_key<AS>(L, key[b], xw, zw, fv);
                i64 p = o + (inc - c);
                for (u32 ph = 0; ph < 2; ++ph) {
                    if (!(ph ? k1b : k0b)) continue;
                    if (p >= out.capacity) {
                        raise_status(status, PL_ERR_CAPACITY);
                        break;
                    }
#pragma unroll
                    for (int w = 0; w < AS; ++w) {
                        out.x[(i64)w * out.capacity + p] = xw[w];
                        out.z[(i64)w * out.capacity + p] = zw[w];
                    }
                    out.f[p] = (u8)ph;
                    out.v[p] = ph ? v[b].y : v[b].x;
                    ++p;
                }
            }
            o += tot;
        }
    }
}

// Filters decided by the fold (segflag 1 = kept): each tile writes at the
// offset k_tile_scan gave it.  Warp-striped items; all flags are loaded
// before any value so the loads overlap.
template <int AS, class Src>
__global__ void __launch_bounds__(kThreads)
    k_emit_counted(Src src, KeyLayout L, const u64* keys, const u32* pay, const double* segval,
                   const u8* segflag, u32 n, const u32* tile_off, int mode, SoAOut out,
                   int* status) {
    __shared__ u32 swarp[kWarps];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const u32 tile = blockIdx.x;
    const u32 wbase = tile * kETile + (u32)warp * (kEItems * 32);
    u32 keepmask = 0;
#pragma unroll
    for (int t = 0; t < kEItems; ++t) {
        const u32 e = wbase + t * 32 + lane;
        if (e < n && segflag[e] == 1) keepmask |= 1u << t;
    }
    double v[kEItems];
    u64 kk[kEItems];
#pragma unroll
    for (int t = 0; t < kEItems; ++t) {
        const bool k = (keepmask >> t) & 1u;
        v[t] = k ? segval[wbase + t * 32 + lane] : 0.0;
        kk[t] = k ? keys[wbase + t * 32 + lane] : 0ull;
    }
    u32 wcount = 0;
    u32 myoff[kEItems];
#pragma unroll
    for (int t = 0; t < kEItems; ++t) {
        const u32 bal = __ballot_sync(0xffffffffu, (keepmask >> t) & 1u);
        myoff[t] = wcount + __popc(bal & lanemask_lt());
        wcount += __popc(bal);
    }
    u32 total;
    const u32 wexcl = block_excl_scan(lane == 0 ? wcount : 0u, swarp, total);
    const u32 base_o = tile_off[tile] + __shfl_sync(0xffffffffu, wexcl, 0);
#pragma unroll
    for (int t = 0; t < kEItems; ++t)
        if ((keepmask >> t) & 1u)
            emit_term<AS>(src, L, kk[t], pay, wbase + t * 32 + lane, mode, v[t],
                          (i64)base_o + myoff[t], out, status);
}

// All filters here (the weight filter needs the unpacked key), with a
// decoupled look-back across tiles for the output offsets.  counters: [3]
// tile counter.
template <int AS, class Src>
__global__ void __launch_bounds__(kThreads) k_emit(Src src, KeyLayout L, const u64* keys,
                                                   const u32* pay, const double* segval,
                                                   const u8* segflag, u32 n, u32* counters,
                                                   u32* lb, int mode, double cutoff,
                                                   u64 max_weight, SoAOut out, i64* d_out_count,
                                                   int* status) {
    __shared__ SegSmem S;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) S.tile = atomicAdd(&counters[3], 1u);
    __syncthreads();
    const u32 tile = S.tile;
    const u32 wbase = tile * kETile + (u32)warp * (kEItems * 32);
    u32 headmask = 0;
#pragma unroll
    for (int t = 0; t < kEItems; ++t) {
        const u32 e = wbase + t * 32 + lane;
        if (e < n && segflag[e]) headmask |= 1u << t;
    }
    double v[kEItems];
    u64 kk[kEItems];
#pragma unroll
    for (int t = 0; t < kEItems; ++t) {
        const bool hd = (headmask >> t) & 1u;
        v[t] = hd ? segval[wbase + t * 32 + lane] : 0.0;
        kk[t] = hd ? keys[wbase + t * 32 + lane] : 0ull;
    }
    u32 keepmask = 0, wcount = 0;
    u32 myoff[kEItems];
#pragma unroll
    for (int t = 0; t < kEItems; ++t) {
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
    for (int t = 0; t < kEItems; ++t)
        if ((keepmask >> t) & 1u)
            emit_term<AS>(src, L, kk[t], pay, wbase + t * 32 + lane, mode, v[t],
                          (i64)base_o + myoff[t], out, status);
    if (tile == gridDim.x - 1 && tid == 0) *d_out_count = (i64)S.excl + total;
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
inline size_t al(size_t b) { return (b + 255) & ~size_t(255); }
// counters: [2] pending segments, [3] emit tiles, [8 + p] tile counter of
// digit pass p; then the operand histograms of a product (kHistScratch,
// 16 * kRadix words); the last word is the windowed-key check.
constexpr int kHistScratch = 8 + kMaxPasses;
constexpr int kCounterWords = kHistScratch + 16 * kRadixW + 8;

// Bump allocator over the workspace; with base == nullptr it only measures.
struct Carve {
    unsigned char* base;
    size_t bytes;
    size_t used = 0;
    template <class T>
    T* take(size_t count) {
        const size_t b = al(sizeof(T) * (count ? count : 1));
        T* r = base ? reinterpret_cast<T*>(base + used) : nullptr;
        used += b;
        return r;
    }
    bool ok() const { return used <= bytes; }
};

int max_chunks(int as) { return (128 * as + 2 + 63) / 64; }

struct Bufs {
    u64 *ka, *kb, *planes;
    u32 *pa, *pb, *hist, *lb, *lb2, *counters;  // lb / lb2: look-back words of even / odd passes
    u8* segflag;
    double *seg_sum, *sv;
    u32 *wfirst, *long_list;
    double2 *rpre, *ptail;
    u32 *tile_kept, *tile_off, *lb_emit;
    u32 *rng_heads, *rng_kept, *rng_off;  // per fold range (index-packed path)
    u64 *orm, *andm;
    i64* d_count;
    int* d_status;
    size_t planes_bytes;
};

void carve_all(Carve& c, i64 n, int nch, Bufs& B) {
    const i64 rtiles = (n + kRTileMin - 1) / kRTileMin + 1;
    const i64 etiles = (n + kETile - 1) / kETile + 1;
    const i64 ngw = (n + kFoldSpan - 1) / kFoldSpan + 16;  // fold ranges; also bounds pending runs
    B.ka = c.take<u64>(n);
    B.kb = c.take<u64>(n);
    B.pa = c.take<u32>(n);
    B.pb = c.take<u32>(n);
    B.sv = c.take<double>(n);
    B.planes = c.take<u64>(nch > 1 ? (size_t)n * nch : 1);
    B.planes_bytes = sizeof(u64) * (nch > 1 ? (size_t)n * nch : 1);
    B.hist = c.take<u32>(kMaxPasses * kRadix);
    // look-back words: 256 per tile of >= 2048 keys, or 1024 per tile of >= 3072
    // keys (10-bit digits)
    const size_t lbw = std::max<size_t>((size_t)rtiles * kRadix,
                                        (size_t)((n + 3071) / 3072 + 1) * kRadixW);
    B.lb = c.take<u32>(lbw);
    B.lb2 = c.take<u32>(lbw);
    B.segflag = c.take<u8>(n + 16);
    B.seg_sum = c.take<double>(n);
    B.wfirst = c.take<u32>(ngw);
    B.long_list = c.take<u32>(ngw);
    B.rpre = c.take<double2>(ngw);
    B.ptail = c.take<double2>(ngw);
    B.tile_kept = c.take<u32>(etiles);
    B.tile_off = c.take<u32>(etiles);
    B.lb_emit = c.take<u32>(etiles);
    B.rng_heads = c.take<u32>(ngw);
    B.rng_kept = c.take<u32>(ngw);
    B.rng_off = c.take<u32>(ngw);
    B.counters = c.take<u32>(kCounterWords);
    B.orm = c.take<u64>(2 * kMaxFields);   // one set per operand of a product
    B.andm = c.take<u64>(2 * kMaxFields);
    B.d_count = c.take<i64>(1);
    B.d_status = c.take<int>(1);
}

size_t ws_for(int, i64 n, int nch) {
    Carve c{nullptr, ~size_t(0)};
    Bufs B;
    carve_all(c, n, nch, B);
    return c.used + 1024;
}

bool carve(void* ws, size_t bytes, i64 n, int nch, Bufs& B) {
    Carve c{reinterpret_cast<unsigned char*>(ws), bytes};
    carve_all(c, n, nch, B);
    return c.ok();
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

// Index-packed layout (kCanonSplit): the varying x / z bits sit above
// ibits = ceil(log2 n) index bits, the flags stay out of the key, and the
// digit passes cover only the x / z bits (8-bit digits at most).  Sorting
// these words orders terms by (x, z) and, within equal (x, z), by index --
// a stable sort by (x, z).  False when the word would exceed 64 bits or no
// x / z bit varies.
bool build_layout_split(int as, const u64* orm, const u64* andm, u32 n, KeyLayout& L,
                        PassPlan& P, u64& imask, int digit_max = 8) {
    const int nf = 2 * as + 1;
    std::memset(&L, 0, sizeof(L));
    std::memset(&P, 0, sizeof(P));
    int ibits = 1;
    while (ibits < 32 && (1ull << ibits) < (u64)n) ++ibits;
    int xz = 0;
    for (int f = 0; f < 2 * as; ++f) {
        const u64 var = orm[f] ^ andm[f];
        L.cbits[f] = andm[f];
        if (var == 0) continue;
        const int lo = __builtin_ctzll(var), hi = 63 - __builtin_clzll(var);
        L.lo[f] = lo;
        L.width[f] = hi - lo + 1;
        xz += L.width[f];
    }
    if (xz == 0 || xz + ibits > 64) return false;
    int off = ibits;
    for (int f = nf - 1; f >= 0; --f) {
        L.off[f] = off;
        off += L.width[f];
    }
    L.total_bits = off;
    L.nchunks = 1;
    L.seg_mask0 = ~1ull;  // bit 0 carries the phase once the last pass has run
    const int passes = (xz + digit_max - 1) / digit_max;
    const int dw = (xz + passes - 1) / passes;
    int np = 0;
    for (int p = 0; p < passes; ++p) {
        P.chunk[np] = 0;
        P.shift[np] = ibits + p * dw;
        P.bits[np] = std::min(dw, xz - p * dw);
        ++np;
    }
    P.first[0] = 0;
    P.first[1] = np;
    P.npasses = np;
    imask = (1ull << ibits) - 1ull;
    return true;
}

// Segment sums: the warp fold, then the carry pass for the segments still
// open after their range and its lookahead.
template <int MODE, class G = NoGather>
int fold_segments(const SegCtx& C, Bufs& B, const FoldFilter& F, int nsm, cudaStream_t st,
                  G g = G{}) {
    const u32 n = C.n;
    const u32 ngw = (n + kFoldSpan - 1) / kFoldSpan;
    const u32 fold_blocks = (ngw + kFoldWarps - 1) / kFoldWarps;
    PL_CUDA_TRY(cudaFuncSetAttribute(k_fold<MODE, G>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFoldSmem));
    // six CTAs (24 warps) per SM: 6 x 37 KB of staging
    PL_CUDA_TRY(cudaFuncSetAttribute(k_fold<MODE, G>,
                                     cudaFuncAttributePreferredSharedMemoryCarveout,
                                     cudaSharedmemCarveoutMaxShared));
    k_fold<MODE, G><<<fold_blocks, 32 * kFoldWarps, kFoldSmem, st>>>(
        C, B.seg_sum, B.segflag, B.wfirst, B.long_list, B.counters, F, g), pl::note_launch();
    // at most one pending segment per fold range
    if constexpr (MODE == kCanonSplit) {
        // ... and the tile scan in the last block (counters[4]: zeroed at the
        // start of the call)
        const int cw = (int)std::max<u32>(1u, std::min<u32>((ngw + 31) / 32, (u32)nsm));
        k_fold_carry<MODE, true><<<cw, 1024, 0, st>>>(B.wfirst, ngw, B.long_list, B.counters,
                                                       B.seg_sum, B.segflag, F, B.rng_off,
                                                       B.d_count, B.counters + 4),
            pl::note_launch();
    } else {
        const int cw_blocks = (int)std::min<u32>((ngw + 7) / 8, (u32)nsm * 4);
        k_fold_carry<MODE><<<cw_blocks, 256, 0, st>>>(B.wfirst, ngw, B.long_list, B.counters,
                                                      B.seg_sum, B.segflag, F),
            pl::note_launch();
    }
    return PL_OK;
}

// Histograms that can be derived instead of counted: none for a plain sum.
template <int AS>
u32 derive_histograms(const SoASrc<AS>&, const KeyLayout&, const PassPlan&, Bufs&, cudaStream_t,
                      bool* scanned, u64* = nullptr, int = kRadix, bool = false) {
    *scanned = false;
    return 0u;
}
template <int AS>
u32 derive_histograms(const WinSrc<AS>&, const KeyLayout&, const PassPlan&, Bufs&, cudaStream_t,
                      bool* scanned, u64* = nullptr, int = kRadix, bool = false) {
    *scanned = false;
    return 0u;
}

// Products: chunk-0 passes free of flags bits come from operand histograms.
// When they are all the passes, the convolution also writes the bucket
// starts and *scanned is set (no k_scan_buckets needed).
template <int AS>
u32 derive_histograms(const ProdSrc<AS>& src, const KeyLayout& L, const PassPlan& P, Bufs& B,
                      cudaStream_t st, bool* scanned, u64* opk = nullptr, int R = kRadix,
                      bool prefilled = false) {
    *scanned = false;
    const int np0 = P.first[1] - P.first[0];
    const int wf = L.width[2 * AS];  // the flags field occupies packed bits [0, wf)
    u32 mask = 0;
    for (int p = 0; p < np0; ++p)
        if (P.shift[p] >= wf) mask |= 1u << p;
    if (!mask) return 0u;
    // scratch after the pass counters: 8 passes x R bins per operand (R =
    // 1024: at most 4 passes, 4 x R)
    u32* hA = B.counters + kHistScratch;
    u32* hB = hA + (R == kRadix ? 8 : 4) * R;
    if (!prefilled &&
        fill32_async(hA, 0u, sizeof(u32) * (R == kRadix ? 16 : 8) * R, st) != cudaSuccess)
        return 0u;
    const SoASrc<AS> a{src.ax, src.az, src.af, src.av, src.sa};
    const SoASrc<AS> b{src.bx, src.bz, src.bf, src.bv, src.sb};
    const dim3 g(grid_for(std::max(src.n, src.m), 256, 64), 2);
    const bool all = np0 == P.npasses && mask == (1u << np0) - 1u;
    if (R == kRadixW) {
        if (!all || np0 > 4) return 0u;  // 10-bit digits need every histogram derived
        k_operand_hist<AS, kRadixW><<<g, 256, 0, st>>>(a, src.n, hA, b, src.m, hB, L, P, mask,
                                                       opk),
            pl::note_launch();
        k_xor_conv<kRadixW><<<np0, kRadixW, 0, st>>>(hA, hB, P, mask, B.hist, 1),
            pl::note_launch();
    } else {
        k_operand_hist<AS><<<g, 256, 0, st>>>(a, src.n, hA, b, src.m, hB, L, P, mask, opk),
            pl::note_launch();
        k_xor_conv<kRadix><<<np0, kRadix, 0, st>>>(hA, hB, P, mask, B.hist, all ? 1 : 0),
            pl::note_launch();
    }
    *scanned = all;
    return mask;
}

// Room for a product's operand packed keys (n_lhs + n_rhs words) in an
// n-word buffer; none for a plain sum.
template <class Src>
bool operand_key_room(const Src&, u32) {
    return false;
}
template <int AS>
bool operand_key_room(const ProdSrc<AS>& src, u32 n) {
    return (u64)src.n + src.m <= (u64)n;
}

// Look-back window of a digit pass (2, 4, 8 or 16; PL_TUNE_RADIX_WINDOW).
// Unset: 8 for index-packed keys (measured best on the product workload), 4
// for key + payload passes.  Returned with the hot polls before a waiting
// thread backs off (PL_TUNE_RADIX_BACKOFF; unset 16 for index-packed keys,
// 64 otherwise) in the bits above 8.
int radix_window(bool konly = false) {
    const long long v = tuning(PL_TUNE_RADIX_WINDOW);
    const int w = (v == 2 || v == 4 || v == 8 || v == 16) ? (int)v : (konly ? 8 : 4);
    const long long b = tuning(PL_TUNE_RADIX_BACKOFF);
    const int hot = (b >= 1 && b <= 1024) ? (int)b : (konly ? 16 : 64);
    return w | (hot << 8);
}

// Keys per thread of a digit pass (8, 12 or 16; PL_TUNE_RADIX_ITEMS).  Unset:
// 12 for index-packed keys (measured best on the product workload), 8 for
// key + payload passes (their 12 extra bytes of shared memory per key).
int radix_items(bool konly = false) {
    const long long v = tuning(PL_TUNE_RADIX_ITEMS);
    if (v == 8 || v == 12 || v == 16) return (int)v;
    return konly ? 12 : 8;
}

// Dynamic shared memory of a digit pass.  (The default carveout is kept:
// the largest one admits more CTAs per SM but leaves the L1 too small for
// the last pass's gathers, and measured slower.)
template <class K>
cudaError_t radix_attrs(K* kernel, int smem) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

// L2 prefetch distance of the digit passes in tiles (PL_TUNE_RADIX_PREFETCH):
// by default one wave -- resident CTAs per SM (looked up once per kernel
// instantiation into `per_sm`) times SMs; -1 off; k > 0 exactly k tiles.
template <class K>
u32 prefetch_ahead(K* kernel, size_t smem, int& per_sm) {
    const long long v = tuning(PL_TUNE_RADIX_PREFETCH);
    if (v < 0) return 0u;
    if (v > 0) return (u32)v;
    if (per_sm == 0) {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, kThreads, smem) !=
                cudaSuccess ||
            b < 1)
            b = 1;
        per_sm = b;
    }
    return (u32)(per_sm * sm_count());
}

template <class Src, int ITEMS>
int radix_pass(bool last, const u64* kin, const u32* vin, u64* kout, u32* vout, u32 n, int shift,
               int bits, const u32* bstart, Bufs& B, u32* lb, u32* lb_next, u32* ctr,
               const Src& src, cudaStream_t st) {
    const u32 tiles = (n + kThreads * ITEMS - 1) / (kThreads * ITEMS);
    const SoASrc<1> nosrc{nullptr, nullptr, nullptr, nullptr, 0};
    const size_t sm = radix_smem(ITEMS);
    static int occ_last = 0, occ_mid = 0;
    if (last) {
        auto* k = k_radix_pass<Src, true, ITEMS, false>;
        PL_CUDA_TRY(radix_attrs(k, (int)sm));
        k<<<tiles, kThreads, sm, st>>>(kin, vin, kout, vout, n, shift, bits, bstart, lb, ctr,
                                       B.d_status, src, B.sv, nullptr, 0ull,
                                       prefetch_ahead(k, sm, occ_last), lb_next, radix_window()),
            pl::note_launch();
    } else {
        auto* k = k_radix_pass<SoASrc<1>, false, ITEMS, false>;
        PL_CUDA_TRY(radix_attrs(k, (int)sm));
        k<<<tiles, kThreads, sm, st>>>(kin, vin, kout, vout, n, shift, bits, bstart, lb, ctr,
                                       B.d_status, nosrc, nullptr, nullptr, 0ull,
                                       prefetch_ahead(k, sm, occ_mid), lb_next, radix_window()),
            pl::note_launch();
    }
    return PL_OK;
}

// 10-bit digit pass over index-packed keys (k_radix_pass_w).
template <class Src, int ITEMS>
int radix_pass_w(bool last, const u64* kin, u64* kout, u32 n, int shift, int bits,
                 const u32* bstart, Bufs& B, u32* lb, u32* lb_next, u32* ctr, const Src& src,
                 const uint2* phs, u64 imask, cudaStream_t st) {
    const u32 tiles = (n + kThreads * ITEMS - 1) / (kThreads * ITEMS);
    const size_t sm = radix_smem_konly(ITEMS);
    static int occ_last = 0, occ_mid = 0;
    if (last) {
        auto* k = k_radix_pass_w<Src, true, ITEMS>;
        PL_CUDA_TRY(radix_attrs(k, (int)sm));
        k<<<tiles, kThreads, sm, st>>>(kin, kout, n, shift, bits, bstart, lb, ctr, B.d_status,
                                       src, B.sv, phs, imask, prefetch_ahead(k, sm, occ_last),
                                       lb_next, radix_window(true)),
            pl::note_launch();
    } else {
        const SoASrc<1> nosrc{nullptr, nullptr, nullptr, nullptr, 0};
        auto* k = k_radix_pass_w<SoASrc<1>, false, ITEMS>;
        PL_CUDA_TRY(radix_attrs(k, (int)sm));
        k<<<tiles, kThreads, sm, st>>>(kin, kout, n, shift, bits, bstart, lb, ctr, B.d_status,
                                       nosrc, nullptr, nullptr, imask,
                                       prefetch_ahead(k, sm, occ_mid), lb_next, radix_window(true)),
            pl::note_launch();
    }
    return PL_OK;
}

template <class S>
struct IsProd : std::false_type {};
template <int AS>
struct IsProd<ProdSrc<AS>> : std::true_type {};

// Digit pass over index-packed keys (no payload).
template <class Src, int ITEMS>
int radix_pass_konly(bool last, const u64* kin, u64* kout, u32 n, int shift, int bits,
                     const u32* bstart, Bufs& B, u32* lb, u32* lb_next, u32* ctr, const Src& src,
                     const uint2* phs, u64 imask, cudaStream_t st) {
    const u32 tiles = (n + kThreads * ITEMS - 1) / (kThreads * ITEMS);
    const size_t sm = radix_smem_konly(ITEMS);
    static int occ_last = 0, occ_mid = 0;
    if (last) {
        auto* k = k_radix_pass<Src, true, ITEMS, true>;
        PL_CUDA_TRY(radix_attrs(k, (int)sm));
        k<<<tiles, kThreads, sm, st>>>(kin, nullptr, kout, nullptr, n, shift, bits, bstart, lb,
                                       ctr, B.d_status, src, B.sv, phs, imask,
                                       prefetch_ahead(k, sm, occ_last), lb_next, radix_window(true)),
            pl::note_launch();
    } else {
        const SoASrc<1> nosrc{nullptr, nullptr, nullptr, nullptr, 0};
        auto* k = k_radix_pass<SoASrc<1>, false, ITEMS, true>;
        PL_CUDA_TRY(radix_attrs(k, (int)sm));
        k<<<tiles, kThreads, sm, st>>>(kin, nullptr, kout, nullptr, n, shift, bits, bstart, lb,
                                       ctr, B.d_status, nosrc, nullptr, nullptr, imask,
                                       prefetch_ahead(k, sm, occ_mid), lb_next, radix_window(true)),
            pl::note_launch();
    }
    return PL_OK;
}

template <int AS, class Src>
int run_collate(const Src& src, u32 n, int mode, const KeyLayout& L, const PassPlan& P,
                const CollateArgs& a, const SoAOut& out, i64* out_count, Bufs& B,
                cudaStream_t st) {
    const int items = radix_items();
    const u32 rtiles = (n + kThreads * items - 1) / (kThreads * items);
    const int nsm = sm_count();
    // the look-back words of the first digit pass; every pass clears the
    // next one's
    const FillReq fr[5] = {{B.hist, 0u, sizeof(u32) * (size_t)std::max(P.npasses, 1) * kRadix},
                           {B.counters, 0u, sizeof(u32) * (size_t)(P.npasses + 8)},
                           {B.d_status, 0u, sizeof(int)},
                           {B.d_count, 0u, sizeof(i64)},
                           {B.lb, 0u, sizeof(u32) * (size_t)rtiles * kRadix}};
    PL_CUDA_TRY(fill32_multi(fr, 5, st));
    const int gblocks = grid_for(n, 256, nsm * 8);
    cudaEvent_t e0 = timed_begin(st);
    bool scanned = false;
    const u32 derived = derive_histograms<AS>(src, L, P, B, st, &scanned);
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
        if (!(c == 0 && scanned)) k_scan_buckets<<<np, kRadix, 0, st>>>(B.hist, p0), pl::note_launch();
        for (int p = p0; p < p0 + np; ++p) {
            cudaEvent_t ev0 = timed_begin(st);
            const bool last = (p == P.npasses - 1);
            const u32* bs = B.hist + (size_t)p * kRadix;
            u32* ctr = B.counters + 8 + p;
            u32* lb = (p & 1) ? B.lb2 : B.lb;
            u32* lbn = (p & 1) ? B.lb : B.lb2;
            int rc = PL_OK;
            if (items == 16)
                rc = radix_pass<Src, 16>(last, kin, vin, kout, vout, n, P.shift[p], P.bits[p], bs,
                                         B, lb, lbn, ctr, src, st);
            else if (items == 12)
                rc = radix_pass<Src, 12>(last, kin, vin, kout, vout, n, P.shift[p], P.bits[p], bs,
                                         B, lb, lbn, ctr, src, st);
            else
                rc = radix_pass<Src, 8>(last, kin, vin, kout, vout, n, P.shift[p], P.bits[p], bs,
                                        B, lb, lbn, ctr, src, st);
            if (rc) return rc;
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
    const u32 etiles = (n + kETile - 1) / kETile;
    // Without a weight filter the fold decides the zero / cutoff filters and
    // counts survivors per emit tile, so the emit needs no look-back.
    const bool counted = a.max_weight == ~0ull;
    const FoldFilter F{counted ? 1 : 0, a.cutoff, B.tile_kept, nullptr, B.rpre, B.ptail,
                       nullptr, nullptr, nullptr};
    if (counted) PL_CUDA_TRY(fill32_async(B.tile_kept, 0u, sizeof(u32) * etiles, st));
    e0 = timed_begin(st);
    int rc = PL_OK;
    if (mode == kCanon) rc = fold_segments<kCanon>(C, B, F, nsm, st);
    else if (mode == kCombine) rc = fold_segments<kCombine>(C, B, F, nsm, st);
    else rc = fold_segments<kProp>(C, B, F, nsm, st);
    if (rc != PL_OK) return rc;
    timed_end(e0, st, "k_fold", 20ull * n);
    e0 = timed_begin(st);
    if (counted) {
        k_tile_scan<<<1, 1024, 0, st>>>(B.tile_kept, etiles, B.tile_off, B.d_count),
            pl::note_launch();
        k_emit_counted<AS, Src><<<etiles, kThreads, 0, st>>>(src, L, kin, vin, B.seg_sum,
                                                             B.segflag, n, B.tile_off, mode, out,
                                                             B.d_status), pl::note_launch();
    } else {
        PL_CUDA_TRY(fill32_async(B.lb_emit, 0u, sizeof(u32) * etiles, st));
        k_emit<AS, Src><<<etiles, kThreads, 0, st>>>(src, L, kin, vin, B.seg_sum, B.segflag, n,
                                                     B.counters, B.lb_emit, mode, a.cutoff,
                                                     a.max_weight, out, B.d_count, B.d_status),
            pl::note_launch();
    }
    timed_end(e0, st, "k_emit", 0ull);
    PL_CUDA_TRY(cudaGetLastError());
    i64 cnt = 0;
    int dstat = 0;
    const ReadReq rr[2] = {{&cnt, B.d_count, sizeof(i64)}, {&dstat, B.d_status, sizeof(int)}};
    PL_CUDA_TRY(readback_sync(rr, 2, st));
    *out_count = cnt;
    if (dstat != 0) return record_status(dstat, "collate: device-side check");
    return PL_OK;
}

// canonicalize() on index-packed keys (layout from build_layout_split;
// filters: zero and cutoff, no weight filter).
// wide: 10-bit digits (a product at >= 12 keys per thread; try_split decides).
template <int AS, class Src>
int run_collate_split(const Src& src, u32 n, const KeyLayout& L, const PassPlan& P, u64 imask,
                      const CollateArgs& a, const SoAOut& out, i64* out_count, Bufs& B,
                      cudaStream_t st, bool wide = false) {
    const int items = radix_items(true);
    const u32 rtiles = (n + kThreads * items - 1) / (kThreads * items);
    const int R = wide ? kRadixW : kRadix;
    const int nsm = sm_count();
    // the chunk-plane buffer is unused with one chunk: phase / sign bit planes,
    // then the (phase-0, phase-1) sums of the segments
    uint2* phs = reinterpret_cast<uint2*>(B.planes);
    double2* seg2 = reinterpret_cast<double2*>(reinterpret_cast<unsigned char*>(B.planes) + al(n));
    // the look-back words of the first digit pass; every pass clears the
    // next one's
    // (and the operand-histogram scratch a product's derived histograms use)
    const FillReq fr[6] = {{B.hist, 0u, sizeof(u32) * (size_t)std::max(P.npasses, 1) * R},
                           {B.counters, 0u, sizeof(u32) * (size_t)(P.npasses + 8)},
                           {B.d_status, 0u, sizeof(int)},
                           {B.d_count, 0u, sizeof(i64)},
                           {B.lb, 0u, sizeof(u32) * (size_t)rtiles * R},
                           {B.counters + kHistScratch, 0u,
                            sizeof(u32) * (size_t)(R == kRadix ? 16 : 8) * R}};
    PL_CUDA_TRY(fill32_multi(fr, 6, st));
    const int gblocks = grid_for(n, 256, nsm * 8);
    cudaEvent_t e0 = timed_begin(st);
    bool scanned = false;
    // a product's operand packed keys go to B.sv, unused until the last
    // digit pass writes the sorted coefficients there
    u64* opk = operand_key_room(src, n) ? reinterpret_cast<u64*>(B.sv) : nullptr;
    const u32 derived = derive_histograms<AS>(src, L, P, B, st, &scanned, opk, R, true);
    if (wide && !scanned) return record_status(PL_ERR_INTERNAL, "collate: 10-bit digit plan");
    timed_end(e0, st, "k_xor_conv", 0ull);
    const u32 count_mask = ~derived & ((1u << P.npasses) - 1u);
    if (!derived) opk = nullptr;  // not written
    e0 = timed_begin(st);
    if (!pack_split_fast<AS>(src, n, L, count_mask, B.ka, phs, opk, st))
        k_pack_split<AS, Src><<<gblocks, 256, 0, st>>>(src, n, L, P, count_mask, B.ka, phs,
                                                       B.hist), pl::note_launch();
    timed_end(e0, st, "k_pack", 8ull * n + n / 4);
    if (!scanned) k_scan_buckets<<<P.npasses, kRadix, 0, st>>>(B.hist, 0), pl::note_launch();
    // a product's fold may take phases and coefficients from the operands
    // itself (PL_TUNE_FOLD_GATHER), so the last digit pass moves keys only
    const bool fold_gather = IsProd<Src>::value && tuning(PL_TUNE_FOLD_GATHER) > 0;
    u64 *kin = B.ka, *kout = B.kb;
    for (int p = 0; p < P.npasses; ++p) {
        cudaEvent_t ev0 = timed_begin(st);
        const bool last = (p == P.npasses - 1) && !fold_gather;
        const u32* bs = B.hist + (size_t)p * R;
        u32* ctr = B.counters + 8 + p;
        u32* lb = (p & 1) ? B.lb2 : B.lb;
        u32* lbn = (p & 1) ? B.lb : B.lb2;
        int rc = PL_OK;
        if (wide) {
            if constexpr (IsProd<Src>::value) {
                if (items == 16)
                    rc = radix_pass_w<Src, 16>(last, kin, kout, n, P.shift[p], P.bits[p], bs, B,
                                               lb, lbn, ctr, src, phs, imask, st);
                else
                    rc = radix_pass_w<Src, 12>(last, kin, kout, n, P.shift[p], P.bits[p], bs, B,
                                               lb, lbn, ctr, src, phs, imask, st);
            } else {
                rc = record_status(PL_ERR_INTERNAL, "collate: 10-bit digits without a product");
            }
        } else if (items == 16)
            rc = radix_pass_konly<Src, 16>(last, kin, kout, n, P.shift[p], P.bits[p], bs, B, lb,
                                           lbn, ctr, src, phs, imask, st);
        else if (items == 12)
            rc = radix_pass_konly<Src, 12>(last, kin, kout, n, P.shift[p], P.bits[p], bs, B, lb,
                                           lbn, ctr, src, phs, imask, st);
        else
            rc = radix_pass_konly<Src, 8>(last, kin, kout, n, P.shift[p], P.bits[p], bs, B, lb,
                                          lbn, ctr, src, phs, imask, st);
        if (rc) return rc;
        // algorithmic bytes: read and write one u64 key per term (+ the two
        // phase / sign bits read and the u64 coefficient written by the last pass)
        timed_end(ev0, st, "k_radix_pass", 16ull * n + (last ? 8ull * n + n / 4 : 0ull));
        std::swap(kin, kout);
    }
    // with the fold gathering, the sorted keys keep their index bits, which
    // segment detection ignores
    SegCtx C{kin, nullptr, B.sv, B.planes, n, 1, fold_gather ? ~imask : L.seg_mask0, kCanon};
    const u32 ngw = (n + kFoldSpan - 1) / kFoldSpan;
    const FoldFilter F{1,      a.cutoff,    nullptr,    seg2,      B.rpre,
                       B.ptail, reinterpret_cast<u64*>(B.seg_sum), B.rng_heads, B.rng_kept};
    e0 = timed_begin(st);
    int rc = PL_OK;
    if constexpr (IsProd<Src>::value) {
        if (fold_gather)
            rc = fold_segments<kCanonSplit>(C, B, F, nsm, st,
                                            ProdGather<AS>{src, phs, imask, n, B.d_status});
        else
            rc = fold_segments<kCanonSplit>(C, B, F, nsm, st);
    } else {
        rc = fold_segments<kCanonSplit>(C, B, F, nsm, st);
    }
    if (rc != PL_OK) return rc;
    timed_end(e0, st, "k_fold", 16ull * n);
    e0 = timed_begin(st);
    // (the tile scan ran in the carry pass's last block)
    k_emit_records<AS><<<(ngw + kWarps - 1) / kWarps, kThreads, 0, st>>>(
        L, reinterpret_cast<const u64*>(B.seg_sum), seg2, B.rng_heads, B.rng_off, ngw, a.cutoff,
        out, B.d_status),
        pl::note_launch();
    timed_end(e0, st, "k_emit", 0ull);
    PL_CUDA_TRY(cudaGetLastError());
    i64 cnt = 0;
    int dstat = 0;
    const ReadReq rr[2] = {{&cnt, B.d_count, sizeof(i64)}, {&dstat, B.d_status, sizeof(int)}};
    PL_CUDA_TRY(readback_sync(rr, 2, st));
    *out_count = cnt;
    if (dstat != 0) return record_status(dstat, "collate: device-side check");
    return PL_OK;
}

// The index-packed path applies to canonicalize() without a weight filter
// whenever the varying (x, z) bits and the index fit one word.
template <int AS, class Src>
bool try_split(const Src& src, u32 n, const u64* orm, const u64* andm, const CollateArgs& a,
               const SoAOut& out, i64* out_count, Bufs& B, cudaStream_t st, int* rc) {
    if (a.mode != kCanon || a.max_weight != ~0ull || tuning(PL_TUNE_INDEX_KEYS) < 0) return false;
    if (B.planes_bytes < al(n) + sizeof(double2) * (size_t)n) return false;
    KeyLayout L;
    PassPlan P;
    u64 imask = 0;
    if (!build_layout_split(AS, orm, andm, n, L, P, imask)) return false;
    // a product (every histogram derived) sorts 10-bit digits where that saves
    // a pass (PL_TUNE_RADIX_WIDE; tiles of >= 12 keys per thread)
    if (IsProd<Src>::value && tuning(PL_TUNE_RADIX_WIDE) > 0 && radix_items(true) >= 12) {
        KeyLayout Lw;
        PassPlan Pw;
        u64 iw = 0;
        if (build_layout_split(AS, orm, andm, n, Lw, Pw, iw, 10) && Pw.npasses < P.npasses &&
            Pw.npasses <= 4) {
            *rc = run_collate_split<AS>(src, n, Lw, Pw, iw, a, out, out_count, B, st, true);
            return true;
        }
    }
    *rc = run_collate_split<AS>(src, n, L, P, imask, a, out, out_count, B, st);
    return true;
}

// The windowed layout (WinSrc) for a wide key: taken when every term fits
// the window form and it needs fewer digit passes than the plain layout
// (canonicalize and sort_and_combine without a weight filter; results are
// identical either way, PL_TUNE_WINDOW_KEYS = -1 switches it off).
template <int AS>
bool try_window(const SoASrc<AS>& src, u32 n, const PassPlan& P0, const CollateArgs& a,
                const SoAOut& out, i64* out_count, Bufs& B, cudaStream_t st, int* rc) {
    if (AS < 2 || P0.npasses <= 16 || a.max_weight != ~0ull || a.mode == kProp ||
        tuning(PL_TUNE_WINDOW_KEYS) < 0)
        return false;
    const WinSrc<AS> ws{src};
    u64* vor = B.orm + kMaxFields;
    u64* vand = B.andm + kMaxFields;
    u32* bad = B.counters + kCounterWords - 1;  // past every pass counter
    const FillReq fm[3] = {{vor, 0u, 8 * kMaxFields},
                           {vand, 0xffffffffu, 8 * kMaxFields},
                           {bad, 0u, sizeof(u32)}};
    cudaError_t e = fill32_multi(fm, 3, st);
    if (e == cudaSuccess) {
        k_win_masks<AS><<<grid_for(n, 256, sm_count() * 4), 256, 0, st>>>(ws, n, a.mode, vor,
                                                                         vand, bad);
        pl::note_launch();
        e = cudaGetLastError();
    }
    u64 hor[kMaxFields], hand[kMaxFields];
    u32 hbad = 1;
    const ReadReq rr[3] = {{hor, vor, 8 * kMaxFields}, {hand, vand, 8 * kMaxFields},
                           {&hbad, bad, sizeof(u32)}};
    if (e == cudaSuccess) e = readback_sync(rr, 3, st);
    if (e != cudaSuccess) {
        *rc = record_cuda(e);
        return true;
    }
    if (hbad) return false;
    KeyLayout L;
    PassPlan P;
    build_layout(AS, a.mode, hor, hand, L, P);
    if (P.npasses >= P0.npasses) return false;
    *rc = run_collate<AS>(ws, n, a.mode, L, P, a, out, out_count, B, st);
    return true;
}

}  // namespace

PL_SPIN_LIMIT_SETTER(set_spin_limit_collate)

// ---------------------------------------------------------------------------
int DevArena::ensure(size_t need) {
    if (need <= bytes) return PL_OK;
    if (ptr) dev_free(ptr, st);
    ptr = nullptr;
    bytes = 0;
    if (dev_alloc(&ptr, need, st) != cudaSuccess) {
        cudaGetLastError();
        return record_status(PL_ERR_OOM, "workspace allocation");
    }
    bytes = need;
    return PL_OK;
}
DevArena::~DevArena() {
    if (ptr) dev_free(ptr, st);
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
        const FillReq fm[2] = {{B.orm, 0u, 8 * kMaxFields}, {B.andm, 0xffffffffu, 8 * kMaxFields}};
        PL_CUDA_TRY(fill32_multi(fm, 2, st));
        k_masks<AS><<<grid_for(n, 256, sm_count() * 4), 256, 0, st>>>(src, n, a.mode, B.orm,
                                                                     B.andm), pl::note_launch();
        u64 hor[kMaxFields], hand[kMaxFields];
        const ReadReq rr[2] = {{hor, B.orm, 8 * kMaxFields}, {hand, B.andm, 8 * kMaxFields}};
        PL_CUDA_TRY(readback_sync(rr, 2, st));
        if (!try_split<AS>(src, n, hor, hand, a, out, out_count, B, st, &rc)) {
            KeyLayout L;
            PassPlan P;
            build_layout(AS, a.mode, hor, hand, L, P);
            if (!try_window<AS>(src, n, P, a, out, out_count, B, st, &rc))
                rc = run_collate<AS>(src, n, a.mode, L, P, a, out, out_count, B, st);
        }
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
        // both operands' OR masks: one launch of per-block partials (no
        // clearing launch), one read-back, reduced here
        u64 hor[2][kMaxFields] = {};
        constexpr int kOrBlocks = 16;
        const SoASrc<AS> sa{lhs.x, lhs.z, lhs.f, lhs.v, lhs.stride};
        const SoASrc<AS> sb{rhs.x, rhs.z, rhs.f, rhs.v, rhs.stride};
        const int gx = grid_for(std::max(lhs.n, rhs.n), 256, kOrBlocks);
        // the operand-histogram scratch, unused until after this read-back
        // (8192 u64 words; the partials take at most 2 x 16 x 32)
        u64* part = reinterpret_cast<u64*>(B.counters + kHistScratch);
        k_operand_or<AS><<<dim3(gx, 2), 256, 0, st>>>(sa, (u32)lhs.n, sb, (u32)rhs.n, part),
            pl::note_launch();
        u64 hpart[2 * kOrBlocks * 2 * AS];
        const ReadReq rr[1] = {{hpart, part, sizeof(u64) * 2 * (size_t)gx * 2 * AS}};
        PL_CUDA_TRY(readback_sync(rr, 1, st));
        for (int w = 0; w < 2; ++w)
            for (int g = 0; g < gx; ++g)
                for (int f = 0; f < 2 * AS; ++f) hor[w][f] |= hpart[(w * gx + g) * 2 * AS + f];
        u64 por[kMaxFields], pand[kMaxFields];
        for (int f = 0; f < 2 * AS; ++f) {
            por[f] = hor[0][f] | hor[1][f];
            pand[f] = 0;
        }
        por[2 * AS] = a.mode == kCanon ? 1ull : 3ull;  // the phase (and sign) may vary
        pand[2 * AS] = 0;
        ProdSrc<AS> src{lhs.x, lhs.z, rhs.x,      rhs.z,      lhs.f,      rhs.f,
                        lhs.v, rhs.v, (u32)lhs.n, (u32)rhs.n, lhs.stride, rhs.stride,
                        FastDiv::make((u32)lhs.n)};
        if (!try_split<AS>(src, n, por, pand, a, out, out_count, B, st, &rc)) {
            KeyLayout L;
            PassPlan P;
            build_layout(AS, a.mode, por, pand, L, P);
            rc = run_collate<AS>(src, n, a.mode, L, P, a, out, out_count, B, st);
        }
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
