/*
 * paulib_oracle.c -- CPU restatement of PauLIB's Pauli-sum hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it, and
 * only as the checker.  The product path (paulib_b200/) never calls it.
 *
 * Every function restates one reference routine in plain, single-threaded C
 * with strict IEEE semantics (built without -ffast-math): coefficient sums
 * run left to right in the order the reference defines, so the results are
 * what the reference's algorithm specifies, independent of OpenMP chunking.
 *
 * Layout: a sum of n terms with AS 64-bit words per string is stored as
 * SoA planes, x[k*n + i] / z[k*n + i] for word k of term i, flags[i]
 * (bit0 = imaginary, bit1 = sign; the exponent k of i^k) and val[i].
 * This is the plane layout of the reference GPU seam
 * (include/gpu/GpuPauliSum.h:8-12).
 *
 * Reference files cited below are paths inside the PauLIB project.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;
typedef uint8_t u8;
typedef int64_t i64;

#define OR_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------ */
/* A growable sum.  The oracle owns its memory; Python reads it back.        */
/* ------------------------------------------------------------------------ */
typedef struct {
    int as;   /* words per string (ceil(N/64)) */
    i64 n;    /* terms */
    i64 cap;  /* capacity in terms */
    u64 *x, *z;
    u8 *f;
    double *v;
} or_sum;

static void sum_reserve(or_sum *s, i64 cap) {
    if (cap <= s->cap) return;
    i64 nc = cap > 2 * s->cap ? cap : 2 * s->cap;
    if (nc < 16) nc = 16;
    u64 *x = (u64 *)calloc((size_t)s->as * nc, sizeof(u64));
    u64 *z = (u64 *)calloc((size_t)s->as * nc, sizeof(u64));
    u8 *f = (u8 *)calloc((size_t)nc, 1);
    double *v = (double *)calloc((size_t)nc, sizeof(double));
    for (int k = 0; k < s->as; ++k) {
        if (s->n) {
            memcpy(x + (size_t)k * nc, s->x + (size_t)k * s->cap, (size_t)s->n * 8);
            memcpy(z + (size_t)k * nc, s->z + (size_t)k * s->cap, (size_t)s->n * 8);
        }
    }
    if (s->n) {
        memcpy(f, s->f, (size_t)s->n);
        memcpy(v, s->v, (size_t)s->n * 8);
    }
    free(s->x); free(s->z); free(s->f); free(s->v);
    s->x = x; s->z = z; s->f = f; s->v = v; s->cap = nc;
}

#define SX(s, k, i) ((s)->x[(size_t)(k) * (s)->cap + (i)])
#define SZ(s, k, i) ((s)->z[(size_t)(k) * (s)->cap + (i)])

OR_EXPORT or_sum *or_sum_new(int as, const u64 *x, const u64 *z, const u8 *f,
                             const double *v, i64 n) {
    or_sum *s = (or_sum *)calloc(1, sizeof(or_sum));
    s->as = as;
    sum_reserve(s, n > 0 ? n : 1);
    for (int k = 0; k < as; ++k)
        for (i64 i = 0; i < n; ++i) {
            SX(s, k, i) = x[(size_t)k * n + i];
            SZ(s, k, i) = z[(size_t)k * n + i];
        }
    if (n) {
        memcpy(s->f, f, (size_t)n);
        memcpy(s->v, v, (size_t)n * 8);
    }
    s->n = n;
    return s;
}

OR_EXPORT void or_sum_free(or_sum *s) {
    if (!s) return;
    free(s->x); free(s->z); free(s->f); free(s->v); free(s);
}

OR_EXPORT i64 or_sum_len(const or_sum *s) { return s->n; }

OR_EXPORT void or_sum_get(const or_sum *s, u64 *x, u64 *z, u8 *f, double *v) {
    for (int k = 0; k < s->as; ++k)
        for (i64 i = 0; i < s->n; ++i) {
            x[(size_t)k * s->n + i] = SX(s, k, i);
            z[(size_t)k * s->n + i] = SZ(s, k, i);
        }
    if (s->n) {
        memcpy(f, s->f, (size_t)s->n);
        memcpy(v, s->v, (size_t)s->n * 8);
    }
}

/* ------------------------------------------------------------------------ */
/* Symplectic product of two strings.                                        */
/* PauliString::multiply (PauliStringCore.h:150-174) and the per-term form   */
/* PauliSum::multiply(i, ps) (PauliSumOperations.h:186-209): per word        */
/*   xbz = ox & bz; anti = (bx & oz) ^ xbz;                                   */
/*   c2 ^= (c1 ^ ox ^ oz ^ bx ^ bz ^ xbz) & anti; c1 ^= anti;                */
/* flags = (fa + fb + popcount(c1) + 2*parity(c2)) mod 4.                    */
/* ------------------------------------------------------------------------ */
static inline u8 mul_words(int as, const u64 *ax, i64 sa, const u64 *az,
                           const u64 *bx, i64 sb, const u64 *bz, u64 *ox,
                           i64 so, u64 *oz, u8 fa, u8 fb) {
    u64 c1 = 0, c2 = 0;
    for (int k = 0; k < as; ++k) {
        const u64 oxk = ax[k * sa], ozk = az[k * sa];
        const u64 bxk = bx[k * sb], bzk = bz[k * sb];
        ox[k * so] = oxk ^ bxk;
        oz[k * so] = ozk ^ bzk;
        const u64 xbz = oxk & bzk;
        const u64 anti = (bxk & ozk) ^ xbz;
        c2 ^= (c1 ^ oxk ^ ozk ^ bxk ^ bzk ^ xbz) & anti;
        c1 ^= anti;
    }
    return (u8)((fa + fb + __builtin_popcountll(c1) + 2 * __builtin_parityll(c2)) & 3);
}

/* inner_product / commute (PauliStringCore.h:126-146): parity of
 * sum_k (ax & bz) ^ (az & bx); 0 means the strings commute. */
static inline int anticommute_words(int as, const u64 *ax, i64 sa, const u64 *az,
                                    const u64 *bx, i64 sb, const u64 *bz) {
    u64 t = 0;
    for (int k = 0; k < as; ++k) t ^= (ax[k * sa] & bz[k * sb]) ^ (az[k * sa] & bx[k * sb]);
    return __builtin_parityll(t);
}

/* ------------------------------------------------------------------------ */
/* Outer product, PauliSum::multiply(rhs) (PauliSumOperations.h:256-306):    */
/* out[i*n + j] = lhs[j] * rhs[i], value lhs_j * rhs_i.                       */
/* ------------------------------------------------------------------------ */
OR_EXPORT or_sum *or_multiply(const or_sum *a, const or_sum *b) {
    const int as = a->as;
    const i64 n = a->n, m = b->n;
    or_sum *o = (or_sum *)calloc(1, sizeof(or_sum));
    o->as = as;
    sum_reserve(o, n * m > 0 ? n * m : 1);
    for (i64 i = 0; i < m; ++i)
        for (i64 j = 0; j < n; ++j) {
            const i64 t = i * n + j;
            o->f[t] = mul_words(as, &SX(a, 0, j), a->cap, &SZ(a, 0, j), &SX(b, 0, i),
                                b->cap, &SZ(b, 0, i), &SX(o, 0, t), o->cap, &SZ(o, 0, t),
                                a->f[j], b->f[i]);
            o->v[t] = a->v[j] * b->v[i];
        }
    o->n = n * m;
    return o;
}

/* ------------------------------------------------------------------------ */
/* commutator_impl (PauliSumOperations.h:316-346), single-threaded order:    */
/* for i over a, for j over b: anticommuting pairs emit a_i*b_j with value   */
/* (2*a_i)*b_j; i[A,B] adds 1 to the phase exponent.                          */
/* ------------------------------------------------------------------------ */
OR_EXPORT or_sum *or_commutator(const or_sum *a, const or_sum *b, int mul_i) {
    const int as = a->as;
    or_sum *o = (or_sum *)calloc(1, sizeof(or_sum));
    o->as = as;
    sum_reserve(o, 16);
    for (i64 i = 0; i < a->n; ++i)
        for (i64 j = 0; j < b->n; ++j) {
            if (!anticommute_words(as, &SX(a, 0, i), a->cap, &SZ(a, 0, i), &SX(b, 0, j),
                                   b->cap, &SZ(b, 0, j)))
                continue;
            if (o->n == o->cap) sum_reserve(o, o->cap * 2);
            const i64 t = o->n;
            u8 fl = mul_words(as, &SX(a, 0, i), a->cap, &SZ(a, 0, i), &SX(b, 0, j), b->cap,
                              &SZ(b, 0, j), &SX(o, 0, t), o->cap, &SZ(o, 0, t), a->f[i],
                              b->f[j]);
            if (mul_i) fl = (u8)((fl + 1) & 3);
            o->f[t] = fl;
            o->v[t] = 2.0 * a->v[i] * b->v[j];
            o->n++;
        }
    return o;
}

/* ------------------------------------------------------------------------ */
/* sort_and_combine (PauliSumOperations.h:369-461).                           */
/* Key: x[0..AS) then z[0..AS) then flags, each compared as unsigned          */
/* (:376-386).  The sort is stable (fixed-chunk stable_sort + stable merges,  */
/* :389-411), so equal keys keep index order and each segment is summed      */
/* left to right from 0.0 (:441-455).  Zero sums are kept.                    */
/* ------------------------------------------------------------------------ */
static const or_sum *g_cmp_sum;
static int key_cmp(i64 a, i64 b) {
    const or_sum *s = g_cmp_sum;
    for (int k = 0; k < s->as; ++k) {
        u64 xa = SX(s, k, a), xb = SX(s, k, b);
        if (xa != xb) return xa < xb ? -1 : 1;
    }
    for (int k = 0; k < s->as; ++k) {
        u64 za = SZ(s, k, a), zb = SZ(s, k, b);
        if (za != zb) return za < zb ? -1 : 1;
    }
    if (s->f[a] != s->f[b]) return s->f[a] < s->f[b] ? -1 : 1;
    return 0;
}

/* Stable bottom-up merge sort of an index array. */
static void stable_sort_idx(i64 *idx, i64 n) {
    i64 *tmp = (i64 *)malloc((size_t)(n > 0 ? n : 1) * sizeof(i64));
    for (i64 w = 1; w < n; w *= 2) {
        for (i64 lo = 0; lo < n; lo += 2 * w) {
            i64 mid = lo + w < n ? lo + w : n;
            i64 hi = lo + 2 * w < n ? lo + 2 * w : n;
            i64 p = lo, q = mid, o = lo;
            while (p < mid && q < hi) {
                if (key_cmp(idx[q], idx[p]) < 0) tmp[o++] = idx[q++];
                else tmp[o++] = idx[p++];
            }
            while (p < mid) tmp[o++] = idx[p++];
            while (q < hi) tmp[o++] = idx[q++];
        }
        memcpy(idx, tmp, (size_t)n * sizeof(i64));
    }
    free(tmp);
}

OR_EXPORT void or_sort_and_combine(or_sum *s) {
    const i64 n = s->n;
    if (n == 0) return;
    i64 *idx = (i64 *)malloc((size_t)n * sizeof(i64));
    for (i64 i = 0; i < n; ++i) idx[i] = i;
    g_cmp_sum = s;
    stable_sort_idx(idx, n);
    or_sum *o = (or_sum *)calloc(1, sizeof(or_sum));
    o->as = s->as;
    sum_reserve(o, n);
    i64 m = 0;
    i64 i = 0;
    while (i < n) {
        const i64 first = idx[i];
        i64 e = i + 1;
        while (e < n && key_cmp(idx[e], first) == 0) ++e;
        double acc = 0.0;
        for (i64 t = i; t < e; ++t) acc += s->v[idx[t]];
        for (int k = 0; k < s->as; ++k) {
            SX(o, k, m) = SX(s, k, first);
            SZ(o, k, m) = SZ(s, k, first);
        }
        o->f[m] = s->f[first];
        o->v[m] = acc;
        ++m;
        i = e;
    }
    o->n = m;
    free(idx);
    /* swap storage */
    free(s->x); free(s->z); free(s->f); free(s->v);
    s->x = o->x; s->z = o->z; s->f = o->f; s->v = o->v; s->cap = o->cap; s->n = m;
    free(o);
}

/* compact(keep_mask) (PauliSumUtils.h:287-308): order-preserving removal. */
static void compact(or_sum *s, const u8 *keep) {
    i64 w = 0;
    for (i64 i = 0; i < s->n; ++i) {
        if (!keep[i]) continue;
        if (w != i) {
            for (int k = 0; k < s->as; ++k) {
                SX(s, k, w) = SX(s, k, i);
                SZ(s, k, w) = SZ(s, k, i);
            }
            s->f[w] = s->f[i];
            s->v[w] = s->v[i];
        }
        ++w;
    }
    s->n = w;
}

/* canonicalize (PauliSumUtils.h:315-328): fold the sign bit into the value,
 * sort_and_combine, drop exact zeros. */
OR_EXPORT void or_canonicalize(or_sum *s) {
    for (i64 i = 0; i < s->n; ++i)
        if (s->f[i] & 2) {
            s->f[i] ^= 2;
            s->v[i] = -s->v[i];
        }
    or_sort_and_combine(s);
    u8 *keep = (u8 *)malloc((size_t)(s->n > 0 ? s->n : 1));
    for (i64 i = 0; i < s->n; ++i) keep[i] = (s->v[i] != 0.0);
    compact(s, keep);
    free(keep);
}

/* cutoff(eps) (PauliSumUtils.h:378-384): keep |c| >= eps. */
OR_EXPORT void or_cutoff(or_sum *s, double eps) {
    u8 *keep = (u8 *)malloc((size_t)(s->n > 0 ? s->n : 1));
    for (i64 i = 0; i < s->n; ++i) keep[i] = (fabs(s->v[i]) >= eps);
    compact(s, keep);
    free(keep);
}

/* term_weight (PauliSumUtils.h:278-283): sum_k popcount(x_k | z_k). */
static i64 term_weight(const or_sum *s, i64 i) {
    i64 w = 0;
    for (int k = 0; k < s->as; ++k) w += __builtin_popcountll(SX(s, k, i) | SZ(s, k, i));
    return w;
}

/* truncate_weight(w) (PauliSumUtils.h:387-393). */
OR_EXPORT void or_truncate_weight(or_sum *s, u64 max_weight) {
    u8 *keep = (u8 *)malloc((size_t)(s->n > 0 ? s->n : 1));
    for (i64 i = 0; i < s->n; ++i) keep[i] = ((u64)term_weight(s, i) <= max_weight);
    compact(s, keep);
    free(keep);
}

/* apply_CNOT(c, t) (PauliSumClifford.h:213-239):
 * flags ^= (xc & zt & (1 ^ xt ^ zc)) << 1;  x_t ^= x_c;  z_c ^= z_t. */
OR_EXPORT void or_apply_cnot(or_sum *s, u64 c, u64 t) {
    const int wc = (int)(c / 64), wt = (int)(t / 64);
    const u64 mc = 1ull << (c % 64), mt = 1ull << (t % 64);
    for (i64 i = 0; i < s->n; ++i) {
        const u64 xc = (SX(s, wc, i) & mc) != 0;
        const u64 zc = (SZ(s, wc, i) & mc) != 0;
        const u64 xt = (SX(s, wt, i) & mt) != 0;
        const u64 zt = (SZ(s, wt, i) & mt) != 0;
        s->f[i] ^= (u8)((xc & zt & (1 ^ xt ^ zc)) << 1);
        SX(s, wt, i) ^= (0 - xc) & mt;
        SZ(s, wc, i) ^= (0 - zt) & mc;
    }
}

/* Bulk Clifford gates (PauliSumClifford.h:44-501): a per-term update of the
 * Pauli bits of qubit c (and t) and of the sign bit, from the bits before
 * the update.  Gate numbers are the library's PL_GATE_* values. */
enum {
    OG_H = 1, OG_S, OG_H_YZ, OG_H_XY, OG_SQRT_X, OG_SQRT_Y, OG_X, OG_Y, OG_Z, OG_I,
    OG_CNOT, OG_CZ, OG_CY, OG_XC_X, OG_XC_Y, OG_XC_Z, OG_YC_X, OG_YC_Y, OG_YC_Z, OG_SWAP,
    OG_ISWAP
};

/* Returns the sign flip; updates the bits in place (b[0..3] = xc, zc, xt, zt). */
static unsigned gate_bits(int g, unsigned *b) {
    const unsigned xc = b[0], zc = b[1], xt = b[2], zt = b[3];
    unsigned sg = 0;
    switch (g) {
    case OG_H:      sg = xc & zc;        b[0] = zc; b[1] = xc; break;          /* :44-62 */
    case OG_S:      sg = xc & zc;        b[1] = zc ^ xc; break;                /* :65-81 */
    case OG_H_YZ:   sg = xc & !zc;       b[0] = xc ^ zc; break;                /* :84-100 */
    case OG_H_XY:   sg = !xc & zc;       b[1] = zc ^ xc; break;                /* :103-119 */
    case OG_SQRT_X: sg = !xc & zc;       b[0] = xc ^ zc; break;                /* :122-138 */
    case OG_SQRT_Y: sg = xc & !zc;       b[0] = zc; b[1] = xc; break;          /* :141-159 */
    case OG_X:      sg = zc; break;                                            /* :162-174 */
    case OG_Y:      sg = xc ^ zc; break;                                       /* :177-190 */
    case OG_Z:      sg = xc; break;                                            /* :193-205 */
    case OG_I:      break;                                                     /* :208-210 */
    case OG_CNOT:   /* :213-239 */
        sg = xc & zt & (1 ^ xt ^ zc); b[2] = xt ^ xc; b[1] = zc ^ zt; break;
    case OG_CZ:     /* :242-267 */
        sg = xc & xt & (zc ^ zt);     b[3] = zt ^ xc; b[1] = zc ^ xt; break;
    case OG_CY: /* :269-295 */
        sg = (xc & zc & zt & !xt) | (xc & xt & !zc & !zt);
        b[1] = zc ^ xt ^ zt; b[2] = xt ^ xc; b[3] = zt ^ xc; break;
    case OG_XC_X: /* :297-322 */
        sg = (xc & zc & zt & !xt) | (xt & zc & zt & !xc);
        b[0] = xc ^ zt; b[2] = xt ^ zc; break;
    case OG_XC_Z: /* :324-349 */
        sg = (xc & xt & zc & zt) | (xt & zc & !xc & !zt);
        b[0] = xc ^ xt; b[3] = zt ^ zc; break;
    case OG_XC_Y: /* :351-377 */
        sg = (xc & xt & zc & !zt) | (zc & zt & !xc & !xt);
        b[0] = xc ^ xt ^ zt; b[2] = xt ^ zc; b[3] = zt ^ zc; break;
    case OG_YC_X: /* :379-405 */
        sg = (xc & xt & zt & !zc) | (zc & zt & !xc & !xt);
        b[0] = xc ^ zt; b[1] = zc ^ zt; b[2] = xt ^ xc ^ zc; break;
    case OG_YC_Z: /* :407-433 */
        sg = (xt & zc & zt & !xc) | (xc & xt & !zc & !zt);
        b[0] = xc ^ xt; b[1] = zc ^ xt; b[3] = zt ^ xc ^ zc; break;
    case OG_YC_Y: /* :435-463 */
        sg = (xc & zt & !xt & !zc) | (xt & zc & !xc & !zt);
        b[0] = xc ^ xt ^ zt; b[1] = zc ^ xt ^ zt; b[2] = xt ^ xc ^ zc; b[3] = zt ^ xc ^ zc;
        break;
    case OG_SWAP:   b[0] = xt; b[1] = zt; b[2] = xc; b[3] = zc; break;        /* :465-490 */
    case OG_ISWAP: {                                      /* :493-499: SWAP, CZ, S(c), S(t) */
        unsigned f = gate_bits(OG_SWAP, b);
        f ^= gate_bits(OG_CZ, b);
        f ^= gate_bits(OG_S, b);
        unsigned u[4] = {b[2], b[3], 0, 0};
        f ^= gate_bits(OG_S, u);
        b[2] = u[0]; b[3] = u[1];
        sg = f; break;
    }
    default: break;
    }
    return sg & 1u;
}

OR_EXPORT int or_apply_clifford(or_sum *s, int gate, u64 c, u64 t) {
    if (gate < OG_H || gate > OG_ISWAP) return -1;
    const int two = gate >= OG_CNOT;
    if (two && c == t) return -1;
    const int wc = (int)(c / 64), wt = (int)(t / 64);
    const u64 mc = 1ull << (c % 64), mt = 1ull << (t % 64);
    for (i64 i = 0; i < s->n; ++i) {
        unsigned b[4] = {(SX(s, wc, i) & mc) != 0, (SZ(s, wc, i) & mc) != 0, 0, 0};
        if (two) { b[2] = (SX(s, wt, i) & mt) != 0; b[3] = (SZ(s, wt, i) & mt) != 0; }
        const unsigned sg = gate_bits(gate, b);
        s->f[i] ^= (u8)(sg << 1);
        SX(s, wc, i) = (SX(s, wc, i) & ~mc) | (b[0] ? mc : 0);
        SZ(s, wc, i) = (SZ(s, wc, i) & ~mc) | (b[1] ? mc : 0);
        if (two) {
            SX(s, wt, i) = (SX(s, wt, i) & ~mt) | (b[2] ? mt : 0);
            SZ(s, wt, i) = (SZ(s, wt, i) & ~mt) | (b[3] ? mt : 0);
        }
    }
    return 0;
}

/* apply_RZ / apply_RX / apply_RY (PauliSumOperations.h:29-104), the gate
 * exp(-i theta/2 P): every term that anticommutes with P_c keeps
 * cos(theta/2) of its value and emits a copy left-multiplied by i P_c
 * (multiply_iZ / iX / iY, PauliSumClifford.h:13-40) with sin(theta/2) of
 * the original value; then `+=` (append + sort_and_combine).  axis: 1 X,
 * 2 Y, 3 Z. */
OR_EXPORT int or_apply_rgate(or_sum *s, int axis, u64 c, double angle) {
    if (axis < 1 || axis > 3) return -1;
    const double ch = cos(angle / 2), sh = sin(angle / 2);
    const int w = (int)(c / 64);
    const u64 mk = 1ull << (c % 64);
    const i64 m = s->n;
    i64 kc = 0;
    for (i64 j = 0; j < m; ++j) {
        const u64 xc = (SX(s, w, j) & mk) != 0, zc = (SZ(s, w, j) & mk) != 0;
        kc += axis == 3 ? xc : axis == 1 ? zc : (xc ^ zc);
    }
    sum_reserve(s, m + kc);
    i64 t = m;
    for (i64 j = 0; j < m; ++j) {
        const u64 xc = (SX(s, w, j) & mk) != 0, zc = (SZ(s, w, j) & mk) != 0;
        const u64 anti = axis == 3 ? xc : axis == 1 ? zc : (xc ^ zc);
        if (!anti) continue;
        const double tv = s->v[j] * sh;
        s->v[j] *= ch;
        for (int k = 0; k < s->as; ++k) { SX(s, k, t) = SX(s, k, j); SZ(s, k, t) = SZ(s, k, j); }
        u8 f = s->f[j];
        if (axis == 3) { f ^= (u8)((!zc) << 1); SZ(s, w, t) ^= mk; }
        else if (axis == 1) { f ^= (u8)(xc << 1); SX(s, w, t) ^= mk; }
        else { f ^= (u8)((!xc) << 1); SX(s, w, t) ^= mk; SZ(s, w, t) ^= mk; }
        s->f[t] = f;
        s->v[t] = tv;
        ++t;
    }
    s->n = t;
    or_sort_and_combine(s);
    return 0;
}

/* basis_state_expectation(bits) (PauliSumUtils.h:178-220): terms with no X
 * bit and a real phase contribute +-value, negated once more per set bit of
 * the basis state under a Z; summed in term order.  bits: AS words. */
OR_EXPORT double or_basis_state_expectation(const or_sum *s, const u64 *bits) {
    double r = 0.0;
    for (i64 i = 0; i < s->n; ++i) {
        int has_x = 0, par = 0;
        for (int k = 0; k < s->as; ++k) {
            has_x |= SX(s, k, i) != 0;
            par ^= __builtin_popcountll(SZ(s, k, i) & bits[k]) & 1;
        }
        if (has_x || (s->f[i] & 1)) continue;
        const double sg = ((s->f[i] & 2) ? -1.0 : 1.0) * (par ? -1.0 : 1.0);
        r += sg * s->v[i];
    }
    return r;
}

/* trace() (PauliSumUtils.h:226-245): 2^nq times the signed sum of the
 * identity terms with a real phase. */
OR_EXPORT double or_trace(const or_sum *s, int nq) {
    double r = 0.0;
    for (i64 i = 0; i < s->n; ++i) {
        int id = 1;
        for (int k = 0; k < s->as; ++k) id &= (SX(s, k, i) | SZ(s, k, i)) == 0;
        if (!id || (s->f[i] & 1)) continue;
        r += ((s->f[i] & 2) ? -1.0 : 1.0) * s->v[i];
    }
    return ldexp(r, nq);
}

/* lookup(ps) (PauliSumUtils.h:246-268): signed sum of the values of the
 * terms with ps's (x, z), phase taken relative to ps's; terms off by +-i
 * are skipped. */
OR_EXPORT double or_lookup(const or_sum *s, const u64 *x, const u64 *z, u8 f) {
    double r = 0.0;
    for (i64 i = 0; i < s->n; ++i) {
        int match = 1;
        for (int k = 0; k < s->as; ++k) match &= SX(s, k, i) == x[k] && SZ(s, k, i) == z[k];
        if (!match) continue;
        const u8 rel = (u8)((s->f[i] - f) & 3);
        if (rel & 1) continue;
        r += (rel & 2) ? -s->v[i] : s->v[i];
    }
    return r;
}

/* frobenius_norm2() (PauliSumUtils.h:400-410): sum of squared values. */
OR_EXPORT double or_frobenius_norm2(const or_sum *s) {
    double r = 0.0;
    for (i64 i = 0; i < s->n; ++i) r += s->v[i] * s->v[i];
    return r;
}

/* trace_product(a, b) (PauliSumUtils.h:412-447): Re tr(A B).  Per (x, z)
 * pattern of A the complex weight sum c i^k is accumulated in A's term
 * order; every term of B with that pattern adds 2^nq Re(w * c_b i^k_b), in
 * B's order (the reference's hash map, restated as a scan). */
OR_EXPORT double or_trace_product(const or_sum *a, const or_sum *b, int nq) {
    double r = 0.0;
    for (i64 j = 0; j < b->n; ++j) {
        double re = 0.0, im = 0.0;
        int found = 0;
        for (i64 i = 0; i < a->n; ++i) {
            int match = 1;
            for (int k = 0; k < a->as; ++k)
                match &= SX(a, k, i) == SX(b, k, j) && SZ(a, k, i) == SZ(b, k, j);
            if (!match) continue;
            found = 1;
            switch (a->f[i] & 3) {
            case 0: re += a->v[i]; break;
            case 1: im += a->v[i]; break;
            case 2: re -= a->v[i]; break;
            default: im -= a->v[i]; break;
            }
        }
        if (!found) continue;
        switch (b->f[j] & 3) {
        case 0: r += re * b->v[j]; break;
        case 1: r -= im * b->v[j]; break;
        case 2: r -= re * b->v[j]; break;
        default: r += im * b->v[j]; break;
        }
    }
    return ldexp(r, nq);
}

/* zero_state_expectation (PauliSumUtils.h:163-177): terms with no X bit and
 * a real phase contribute +-value, summed in term order. */
OR_EXPORT double or_zero_state_expectation(const or_sum *s) {
    double r = 0.0;
    for (i64 i = 0; i < s->n; ++i) {
        int has_x = 0;
        for (int k = 0; k < s->as; ++k)
            if (SX(s, k, i)) { has_x = 1; break; }
        if (has_x) continue;
        if (s->f[i] & 1) continue;
        const double sign = (s->f[i] & 2) ? -1.0 : 1.0;
        r += sign * s->v[i];
    }
    return r;
}

/* isCloseOne (PauliSumOperations.h:19-21). */
static int close_one(double v) { return fabs(v - 1.0) <= 1e-14; }

/* evolve for ONE rotation term (P, theta) (PauliSumOperations.h:107-183).
 * ps = P with its phase bit flipped (ps = iP).  Fast paths at theta ~ 0, pi,
 * +-pi/2; otherwise every anticommuting term j keeps value*cos in place and
 * appends (Q_j * ps, (-sin) * value) in j order, followed by `+=`
 * (append + sort_and_combine, PauliSumCore.h:233-237). */
static void evolve_one(or_sum *s, const u64 *px, const u64 *pz, u8 pf, double theta) {
    const int as = s->as;
    u64 psx[16], psz[16];
    for (int k = 0; k < as; ++k) { psx[k] = px[k]; psz[k] = pz[k]; }
    const u8 psf = pf ^ 1;
    const double c = cos(theta), sn = sin(theta);
    const i64 m = s->n;
    u64 tx[16], tz[16];
    if (close_one(c)) return;
    if (close_one(-c)) {
        for (i64 j = 0; j < m; ++j)
            if (anticommute_words(as, &SX(s, 0, j), s->cap, &SZ(s, 0, j), psx, 1, psz))
                s->f[j] ^= 2;
        return;
    }
    if (close_one(sn) || close_one(-sn)) {
        const int flip = close_one(sn);
        for (i64 j = 0; j < m; ++j) {
            if (!anticommute_words(as, &SX(s, 0, j), s->cap, &SZ(s, 0, j), psx, 1, psz)) continue;
            u8 fj = s->f[j];
            if (flip) fj ^= 2;
            s->f[j] = mul_words(as, &SX(s, 0, j), s->cap, &SZ(s, 0, j), psx, 1, psz, tx, 1, tz,
                                fj, psf);
            for (int k = 0; k < as; ++k) { SX(s, k, j) = tx[k]; SZ(s, k, j) = tz[k]; }
        }
        return;
    }
    /* general branch: count, then append */
    i64 kcount = 0;
    for (i64 j = 0; j < m; ++j)
        kcount += anticommute_words(as, &SX(s, 0, j), s->cap, &SZ(s, 0, j), psx, 1, psz);
    sum_reserve(s, m + kcount);
    i64 t = m;
    for (i64 j = 0; j < m; ++j) {
        if (!anticommute_words(as, &SX(s, 0, j), s->cap, &SZ(s, 0, j), psx, 1, psz)) continue;
        const double orig = s->v[j];
        s->v[j] = orig * c;
        s->f[t] = mul_words(as, &SX(s, 0, j), s->cap, &SZ(s, 0, j), psx, 1, psz, &SX(s, 0, t),
                            s->cap, &SZ(s, 0, t), s->f[j], psf);
        s->v[t] = -sn * orig;
        ++t;
    }
    s->n = t;
    or_sort_and_combine(s);
}

/* PauliSum::evolve(rotations): rotations applied one after another, in
 * order (PauliSumOperations.h:107-110). */
OR_EXPORT void or_evolve(or_sum *s, const or_sum *rot) {
    u64 px[16], pz[16];
    for (i64 r = 0; r < rot->n; ++r) {
        for (int k = 0; k < rot->as; ++k) { px[k] = SX(rot, k, r); pz[k] = SZ(rot, k, r); }
        evolve_one(s, px, pz, rot->f[r], rot->v[r]);
    }
}

/* trim(max_terms) (PauliSumUtils.h:331-345) keeps the max_terms terms of
 * largest |c| via std::nth_element; which of several equal-|c| terms at the
 * boundary survive is up to the library's introselect.  The oracle keeps
 * the largest |c|, breaking ties at the boundary by lower index, and keeps
 * the survivors in their original order. */
static int g_trim_cmp(const void *pa, const void *pb);
static const double *g_trim_v;
static int g_trim_cmp(const void *pa, const void *pb) {
    const i64 a = *(const i64 *)pa, b = *(const i64 *)pb;
    const double fa = fabs(g_trim_v[a]), fb = fabs(g_trim_v[b]);
    if (fa != fb) return fa > fb ? -1 : 1;
    return a < b ? -1 : (a > b);
}
OR_EXPORT void or_trim(or_sum *s, u64 max_terms) {
    if ((u64)s->n <= max_terms) return;
    i64 *idx = (i64 *)malloc((size_t)s->n * sizeof(i64));
    for (i64 i = 0; i < s->n; ++i) idx[i] = i;
    g_trim_v = s->v;
    qsort(idx, (size_t)s->n, sizeof(i64), g_trim_cmp);
    u8 *keep = (u8 *)calloc((size_t)s->n, 1);
    for (u64 i = 0; i < max_terms; ++i) keep[idx[i]] = 1;
    compact(s, keep);
    free(keep);
    free(idx);
}

/* trim(max_terms, keep) (PauliSumUtils.h:347-375): terms whose (x, z)
 * pattern occurs in keep are always kept (the reference's XZ hash set;
 * here a linear scan of the small keep sum); the others compete for what
 * is left of max_terms by |c|, ties to the lower index as in or_trim. */
OR_EXPORT void or_trim_protected(or_sum *s, u64 max_terms, const or_sum *keep) {
    if ((u64)s->n <= max_terms) return;
    const int as = s->as;
    u8 *mask = (u8 *)calloc((size_t)s->n, 1);
    i64 *idx = (i64 *)malloc((size_t)s->n * sizeof(i64));
    i64 m = 0;
    for (i64 i = 0; i < s->n; ++i) {
        int prot = 0;
        for (i64 j = 0; j < keep->n && !prot; ++j) {
            int same = 1;
            for (int k = 0; k < as && same; ++k)
                same = s->x[k * s->cap + i] == keep->x[k * keep->cap + j] &&
                       s->z[k * s->cap + i] == keep->z[k * keep->cap + j];
            prot = same;
        }
        if (prot) mask[i] = 1;
        else idx[m++] = i;
    }
    const u64 protected_count = (u64)(s->n - m);
    const u64 budget = max_terms > protected_count ? max_terms - protected_count : 0;
    g_trim_v = s->v;
    qsort(idx, (size_t)m, sizeof(i64), g_trim_cmp);
    for (i64 i = 0; i < m && (u64)i < budget; ++i) mask[idx[i]] = 1;
    compact(s, mask);
    free(mask);
    free(idx);
}

/* TruncationOptions (PauliPropagation.h:27-31); "disabled" mirrors the
 * reference's SIZE_MAX / 0 sentinels. */
typedef struct {
    u64 max_weight;            /* UINT64_MAX = disabled */
    double coefficient_cutoff; /* <= 0 = disabled */
    u64 max_terms;             /* UINT64_MAX = disabled */
} or_trunc;

/* apply_truncation (PauliPropagation.h:36-47). */
OR_EXPORT void or_apply_truncation(or_sum *s, const or_trunc *o) {
    or_canonicalize(s);
    if (o->max_weight != UINT64_MAX) or_truncate_weight(s, o->max_weight);
    if (o->coefficient_cutoff > 0.0) or_cutoff(s, o->coefficient_cutoff);
    if (o->max_terms != UINT64_MAX) or_trim(s, o->max_terms);
}

/* propagate (PauliPropagation.h:54-63) generalised to a circuit that also
 * contains CNOTs.  ops is a list of int32 triples (kind, a, b), in
 * application order: kind 0 = rotation number a of `rot`, kind 1 = CNOT
 * with control a and target b.  Heisenberg propagation walks the list in
 * reverse; a rotation is evolve + apply_truncation, a CNOT is apply_CNOT
 * (a string bijection, PauliSumClifford.h:213-239) with no truncation.
 * With ops == NULL the circuit is every rotation of `rot` in order, which
 * is exactly the reference's propagate(). */
OR_EXPORT void or_propagate(or_sum *s, const or_sum *rot, const int32_t *ops, i64 n_ops,
                            const or_trunc *o) {
    u64 px[16], pz[16];
    const i64 total = ops ? n_ops : rot->n;
    for (i64 l = total; l-- > 0;) {
        int kind = ops ? ops[3 * l] : 0;
        i64 a = ops ? ops[3 * l + 1] : l;
        if (kind == 1) {
            or_apply_cnot(s, (u64)a, (u64)ops[3 * l + 2]);
            continue;
        }
        if (kind >= 100) { /* Clifford gate kind - 100 on (a, b), no truncation */
            or_apply_clifford(s, kind - 100, (u64)a, (u64)ops[3 * l + 2]);
            continue;
        }
        for (int k = 0; k < rot->as; ++k) { px[k] = SX(rot, k, a); pz[k] = SZ(rot, k, a); }
        evolve_one(s, px, pz, rot->f[a], rot->v[a]);
        or_apply_truncation(s, o);
    }
}
