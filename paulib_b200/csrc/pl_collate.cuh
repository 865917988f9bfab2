// pl_collate.cuh -- internal interface of the collate engine (sort + merge
// of equal keys), shared by the ABI entry points and the propagation state.
#pragma once

#include "pl_common.cuh"

namespace pl {

// How the flags byte enters the key and the merge (see pl_collate.cu).
enum CollateMode : int {
    kCanon = 0,    // canonicalize(): sign folded into the value, key (x,z,phase)
    kCombine = 1,  // sort_and_combine(): key (x,z,flags), value as is, zeros kept
    kProp = 2,     // evolve's `+=` followed by canonicalize(): key (x,z,phase,sign),
                   // merge by (x,z,phase) as S(sign 0) - S(sign 1)
};

struct SoAView {
    const u64* x = nullptr;
    const u64* z = nullptr;
    const u8* f = nullptr;
    const double* v = nullptr;
    i64 n = 0;
    i64 stride = 0;
};

struct SoAOut {
    u64* x = nullptr;
    u64* z = nullptr;
    u8* f = nullptr;
    double* v = nullptr;
    i64 capacity = 0;  // plane stride and maximum term count
};

// Grow-only device arena, allocated in order on its owner's stream.
struct DevArena {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t st = nullptr;
    int ensure(size_t need);
    ~DevArena();
};

struct CollateArgs {
    int mode = kCanon;
    double cutoff = 0.0;           // > 0 enables
    u64 max_weight = ~0ull;        // != ~0 enables
};

// Bytes of workspace a collate of n terms may need.
size_t collate_ws_bytes(int as, i64 n);

// Collate an SoA sum.  Synchronous: on return *out_count holds the output
// size (host).  Output must not alias the input.
int collate_soa(int as, const SoAView& in, const SoAOut& out, const CollateArgs& a,
                i64* out_count, void* ws, size_t ws_bytes, cudaStream_t stream);

// Fused product + collate (lhs * rhs products in i*n + j order).
size_t multiply_collate_ws_bytes(int as, i64 n, i64 m);
int multiply_collate(int as, const SoAView& lhs, const SoAView& rhs, const SoAOut& out,
                     const CollateArgs& a, i64* out_count, void* ws, size_t ws_bytes,
                     cudaStream_t stream);

// Outer product and commutator launchers (pl_terms.cu); s* are plane strides.
int multiply_impl(int as, const u64* ax, const u64* az, const u8* af, const double* av, i64 n,
                  i64 sa, const u64* bx, const u64* bz, const u8* bf, const double* bv, i64 m,
                  i64 sb, u64* ox, u64* oz, u8* of, double* ov, i64 so, cudaStream_t st);
int commutator_impl(int as, int mul_i, const u64* ax, const u64* az, const u8* af,
                    const double* av, i64 n, i64 sa, const u64* bx, const u64* bz, const u8* bf,
                    const double* bv, i64 m, i64 sb, u64* ox, u64* oz, u8* of, double* ov,
                    i64 capacity, unsigned long long* d_count, bool wait, cudaStream_t st);

}  // namespace pl
