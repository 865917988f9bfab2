// ref_shim.cpp -- C ABI over the UNMODIFIED reference headers.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile against the PauLIB
// include/ tree (PauliSum.h + PauliPropagation.h; PauLib.h is avoided
// because it pulls in GSim.h, which needs Eigen) with the reference's own
// flags (-O3 -march=... -ffast-math -fopenmp, CMakeLists.txt:26-29).  The
// library lands in oracle/_ref/ and is used to pin the C restatement
// (oracle/paulib_oracle.c) and as the timed CPU baseline.  Nothing in the
// product path loads it.
//
// The ABI mirrors the oracle's: opaque sum handles holding
// paulib::PauliSum<64*AS, double>, SoA planes x[k*n+i] on the wire.

#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

#include "PauliPropagation.h"
#include "PauliSum.h"

#include <omp.h>

using namespace paulib;
using u64 = std::uint64_t;
using u8 = std::uint8_t;
using i64 = std::int64_t;

namespace {

struct SumBase {
    int as = 1;
    virtual ~SumBase() = default;
    virtual i64 len() const = 0;
    virtual void get(u64* x, u64* z, u8* f, double* v) const = 0;
    virtual void canonicalize() = 0;
    virtual void sort_and_combine() = 0;
    virtual void cutoff(double eps) = 0;
    virtual void truncate_weight(u64 w) = 0;
    virtual void apply_cnot(u64 c, u64 t) = 0;
    virtual double zero_state_expectation() const = 0;
    virtual void evolve(const SumBase* rot) = 0;
    virtual SumBase* multiply(const SumBase* rhs) const = 0;
    virtual SumBase* commutator(const SumBase* rhs, int mul_i) const = 0;
    virtual void propagate(const SumBase* rot, const std::int32_t* ops, i64 n_ops,
                           u64 max_weight, double cutoff, u64 max_terms) = 0;
    virtual void trim(u64 max_terms) = 0;
    virtual void trim_protected(u64 max_terms, const SumBase* keep) = 0;
    virtual int apply_clifford(int gate, u64 c, u64 t) = 0;
    virtual int apply_rgate(int axis, u64 c, double angle) = 0;
    virtual double basis_state_expectation(const char* bits) const = 0;
    virtual double trace() const = 0;
    virtual double frobenius_norm2() const = 0;
    virtual double lookup(const u64* x, const u64* z, u8 f) const = 0;
    virtual double trace_product(const SumBase* b) const = 0;
};

template <std::size_t N>
struct Sum final : SumBase {
    using PS = PauliSum<N, double>;
    static constexpr int AS = (int)PS::ArraySize;
    PS s;

    Sum() { as = AS; }

    void set(const u64* x, const u64* z, const u8* f, const double* v, i64 n) {
        for (int k = 0; k < AS; ++k) {
            s.x_data[k].assign(x + (std::size_t)k * n, x + (std::size_t)k * n + n);
            s.z_data[k].assign(z + (std::size_t)k * n, z + (std::size_t)k * n + n);
        }
        s.flags.assign(f, f + n);
        s.value.assign(v, v + n);
    }
    i64 len() const override { return (i64)s.get_length(); }
    void get(u64* x, u64* z, u8* f, double* v) const override {
        const i64 n = len();
        for (int k = 0; k < AS; ++k) {
            if (n) {
                std::memcpy(x + (std::size_t)k * n, s.x_data[k].data(), (std::size_t)n * 8);
                std::memcpy(z + (std::size_t)k * n, s.z_data[k].data(), (std::size_t)n * 8);
            }
        }
        if (n) {
            std::memcpy(f, s.flags.data(), (std::size_t)n);
            std::memcpy(v, s.value.data(), (std::size_t)n * 8);
        }
    }
    void canonicalize() override { s.canonicalize(); }
    void sort_and_combine() override { s.sort_and_combine(); }
    void cutoff(double eps) override { s.cutoff(eps); }
    void truncate_weight(u64 w) override { s.truncate_weight((std::size_t)w); }
    void apply_cnot(u64 c, u64 t) override { s.apply_CNOT((std::size_t)c, (std::size_t)t); }
    double zero_state_expectation() const override { return s.zero_state_expectation(); }
    void evolve(const SumBase* rot) override { s.evolve(static_cast<const Sum*>(rot)->s); }
    SumBase* multiply(const SumBase* rhs) const override {
        auto* o = new Sum();
        o->s = s;
        o->s.multiply(static_cast<const Sum*>(rhs)->s);
        return o;
    }
    SumBase* commutator(const SumBase* rhs, int mul_i) const override {
        auto* o = new Sum();
        const auto& b = static_cast<const Sum*>(rhs)->s;
        o->s = mul_i ? i_commutator(s, b) : paulib::commutator(s, b);
        return o;
    }
    void trim(u64 max_terms) override { s.trim((std::size_t)max_terms); }
    void trim_protected(u64 max_terms, const SumBase* keep) override {
        s.trim((std::size_t)max_terms, static_cast<const Sum*>(keep)->s);
    }
    // gate numbers: the library's PL_GATE_* values
    int apply_clifford(int gate, u64 c, u64 t) override {
        const std::size_t a = (std::size_t)c, b = (std::size_t)t;
        switch (gate) {
            case 1: s.apply_H(a); break;
            case 2: s.apply_S(a); break;
            case 3: s.apply_H_YZ(a); break;
            case 4: s.apply_H_XY(a); break;
            case 5: s.apply_sqrt_X(a); break;
            case 6: s.apply_sqrt_Y(a); break;
            case 7: s.apply_X(a); break;
            case 8: s.apply_Y(a); break;
            case 9: s.apply_Z(a); break;
            case 10: s.apply_I(a); break;
            case 11: s.apply_CNOT(a, b); break;
            case 12: s.apply_CZ(a, b); break;
            case 13: s.apply_CY(a, b); break;
            case 14: s.apply_XC_X(a, b); break;
            case 15: s.apply_XC_Y(a, b); break;
            case 16: s.apply_XC_Z(a, b); break;
            case 17: s.apply_YC_X(a, b); break;
            case 18: s.apply_YC_Y(a, b); break;
            case 19: s.apply_YC_Z(a, b); break;
            case 20: s.apply_SWAP(a, b); break;
            case 21: s.apply_iSWAP(a, b); break;
            default: return -1;
        }
        return 0;
    }
    // num_qubits_ of these sums is the capacity N = 64 * AS
    double basis_state_expectation(const char* bits) const override {
        return s.basis_state_expectation(std::string(bits));
    }
    double trace() const override { return s.trace(); }
    double frobenius_norm2() const override { return s.frobenius_norm2(); }
    double lookup(const u64* x, const u64* z, u8 f) const override {
        paulib::PauliString<N> ps;
        for (int k = 0; k < AS; ++k) {
            ps.x[k] = (std::size_t)x[k];
            ps.z[k] = (std::size_t)z[k];
        }
        ps.flags = f;
        return s.lookup(ps);
    }
    double trace_product(const SumBase* b) const override {
        return paulib::trace_product(s, static_cast<const Sum*>(b)->s);
    }
    int apply_rgate(int axis, u64 c, double angle) override {
        if (axis == 1) s.apply_RX((std::size_t)c, angle);
        else if (axis == 2) s.apply_RY((std::size_t)c, angle);
        else if (axis == 3) s.apply_RZ((std::size_t)c, angle);
        else return -1;
        return 0;
    }
    void propagate(const SumBase* rotb, const std::int32_t* ops, i64 n_ops, u64 max_weight,
                   double cutoff, u64 max_terms) override {
        const auto& rot = static_cast<const Sum*>(rotb)->s;
        TruncationOptions<double> opts;
        opts.max_weight = max_weight == std::numeric_limits<u64>::max()
                              ? std::numeric_limits<std::size_t>::max()
                              : (std::size_t)max_weight;
        opts.coefficient_cutoff = cutoff;
        opts.max_terms = max_terms == std::numeric_limits<u64>::max()
                             ? std::numeric_limits<std::size_t>::max()
                             : (std::size_t)max_terms;
        if (!ops) {
            paulib::propagate(s, rot, opts);
            return;
        }
        // Circuits with CNOTs: the reference's propagate() takes rotations
        // only, so compose its own primitives exactly as propagate() does per
        // rotation (PauliPropagation.h:54-63) and apply_CNOT per CNOT.
        for (i64 l = n_ops; l-- > 0;) {
            const int kind = ops[3 * l];
            if (kind == 1) {
                s.apply_CNOT((std::size_t)ops[3 * l + 1], (std::size_t)ops[3 * l + 2]);
                continue;
            }
            PauliSum<N, double> gate;
            gate.num_qubits_ = rot.num_qubits();
            gate.push_back(rot.get_pauli_string((std::size_t)ops[3 * l + 1]),
                           rot.value[(std::size_t)ops[3 * l + 1]]);
            s.evolve(gate);
            apply_truncation(s, opts);
        }
    }
};

template <std::size_t N>
SumBase* make(const u64* x, const u64* z, const u8* f, const double* v, i64 n) {
    auto* s = new Sum<N>();
    s->set(x, z, f, v, n);
    return s;
}

template <std::size_t N>
SumBase* make_random(i64 terms, u64 seed, u64 num_qubits) {
    auto* s = new Sum<N>();
    s->s = paulib::random_pauli_sum<N, double>((std::size_t)terms, seed, (std::size_t)num_qubits);
    return s;
}

}  // namespace

extern "C" {

__attribute__((visibility("default"))) void* ref_sum_new(int as, const u64* x, const u64* z,
                                                         const u8* f, const double* v, i64 n) {
    switch (as) {
        case 1: return make<64>(x, z, f, v, n);
        case 2: return make<128>(x, z, f, v, n);
        case 3: return make<192>(x, z, f, v, n);
        case 4: return make<256>(x, z, f, v, n);
        case 8: return make<512>(x, z, f, v, n);
        case 16: return make<1024>(x, z, f, v, n);
        default: return nullptr;
    }
}
// random_pauli_sum (PauliSumUtils.h:114-154) of capacity 64 * as
__attribute__((visibility("default"))) void* ref_random_pauli_sum(int as, i64 terms, u64 seed,
                                                                  u64 num_qubits) {
    switch (as) {
        case 1: return make_random<64>(terms, seed, num_qubits);
        case 2: return make_random<128>(terms, seed, num_qubits);
        case 4: return make_random<256>(terms, seed, num_qubits);
        default: return nullptr;
    }
}
__attribute__((visibility("default"))) void ref_sum_free(void* h) { delete (SumBase*)h; }
__attribute__((visibility("default"))) i64 ref_sum_len(const void* h) {
    return ((const SumBase*)h)->len();
}
__attribute__((visibility("default"))) void ref_sum_get(const void* h, u64* x, u64* z, u8* f,
                                                        double* v) {
    ((const SumBase*)h)->get(x, z, f, v);
}
__attribute__((visibility("default"))) void ref_canonicalize(void* h) {
    ((SumBase*)h)->canonicalize();
}
__attribute__((visibility("default"))) void ref_sort_and_combine(void* h) {
    ((SumBase*)h)->sort_and_combine();
}
__attribute__((visibility("default"))) void ref_cutoff(void* h, double eps) {
    ((SumBase*)h)->cutoff(eps);
}
__attribute__((visibility("default"))) void ref_truncate_weight(void* h, u64 w) {
    ((SumBase*)h)->truncate_weight(w);
}
__attribute__((visibility("default"))) void ref_trim(void* h, u64 m) { ((SumBase*)h)->trim(m); }
__attribute__((visibility("default"))) int ref_apply_clifford(void* h, int g, u64 c, u64 t) {
    return ((SumBase*)h)->apply_clifford(g, c, t);
}
__attribute__((visibility("default"))) int ref_apply_rgate(void* h, int axis, u64 c, double a) {
    return ((SumBase*)h)->apply_rgate(axis, c, a);
}
__attribute__((visibility("default"))) double ref_basis_state_expectation(const void* h,
                                                                         const char* bits) {
    return ((const SumBase*)h)->basis_state_expectation(bits);
}
__attribute__((visibility("default"))) double ref_trace(const void* h) {
    return ((const SumBase*)h)->trace();
}
__attribute__((visibility("default"))) double ref_frobenius_norm2(const void* h) {
    return ((const SumBase*)h)->frobenius_norm2();
}
__attribute__((visibility("default"))) double ref_lookup(const void* h, const u64* x,
                                                         const u64* z, u8 f) {
    return ((const SumBase*)h)->lookup(x, z, f);
}
__attribute__((visibility("default"))) double ref_trace_product(const void* a, const void* b) {
    return ((const SumBase*)a)->trace_product((const SumBase*)b);
}
__attribute__((visibility("default"))) void ref_trim_protected(void* h, u64 m, const void* k) {
    ((SumBase*)h)->trim_protected(m, (const SumBase*)k);
}
__attribute__((visibility("default"))) void ref_apply_cnot(void* h, u64 c, u64 t) {
    ((SumBase*)h)->apply_cnot(c, t);
}
__attribute__((visibility("default"))) double ref_zero_state_expectation(const void* h) {
    return ((const SumBase*)h)->zero_state_expectation();
}
__attribute__((visibility("default"))) void ref_evolve(void* h, const void* rot) {
    ((SumBase*)h)->evolve((const SumBase*)rot);
}
__attribute__((visibility("default"))) void* ref_multiply(const void* a, const void* b) {
    return ((const SumBase*)a)->multiply((const SumBase*)b);
}
__attribute__((visibility("default"))) void* ref_commutator(const void* a, const void* b,
                                                            int mul_i) {
    return ((const SumBase*)a)->commutator((const SumBase*)b, mul_i);
}
__attribute__((visibility("default"))) void ref_propagate(void* h, const void* rot,
                                                          const std::int32_t* ops, i64 n_ops,
                                                          u64 max_weight, double cutoff,
                                                          u64 max_terms) {
    ((SumBase*)h)->propagate((const SumBase*)rot, ops, n_ops, max_weight, cutoff, max_terms);
}
__attribute__((visibility("default"))) int ref_max_threads() { return omp_get_max_threads(); }
__attribute__((visibility("default"))) void ref_set_threads(int n) { omp_set_num_threads(n); }

}  // extern "C"
