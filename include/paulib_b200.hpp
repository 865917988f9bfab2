// paulib_b200.hpp -- C++ facade over the C ABI (paulib_b200.h) with the
// reference's PauliSum<N, double> surface for the hot path: the names,
// argument meanings and exception types of PauLIB's PauliSum
// (PauliSumCore.h, PauliSumOperations.h, PauliSumUtils.h), commutator /
// i_commutator, and propagate / propagate_expectation with
// TruncationOptions (PauliPropagation.h:27-71).
//
// The sum lives in device memory (a pl_state); every method runs on the
// GPU.  The public host planes x_data / z_data / flags / value mirror the
// reference's public fields but are filled only by download() and pushed
// back by upload() -- device-resident sums do not keep a host copy current.
//
// Status codes become exceptions as in the reference: PL_ERR_INVALID_ARG ->
// std::invalid_argument, PL_ERR_OOM -> std::bad_alloc, anything else ->
// std::runtime_error.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <new>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "paulib_b200.h"

namespace paulib_b200 {

inline void check(int status, const char* what) {
    if (status == PL_OK) return;
    const std::string msg = std::string(what) + ": " + pl_last_error_message();
    if (status == PL_ERR_INVALID_ARG) throw std::invalid_argument(msg);
    if (status == PL_ERR_OOM) throw std::bad_alloc();
    throw std::runtime_error(msg);
}

// TruncationOptions<T> (PauliPropagation.h:27-31): SIZE_MAX / 0 disable.
template <typename T = double>
struct TruncationOptions {
    std::size_t max_weight = SIZE_MAX;
    T coefficient_cutoff = T(0);
    std::size_t max_terms = SIZE_MAX;
    pl_truncation c_abi() const {
        pl_truncation t;
        t.max_weight = max_weight == SIZE_MAX ? UINT64_MAX : (uint64_t)max_weight;
        t.coefficient_cutoff = (double)coefficient_cutoff;
        t.max_terms = max_terms == SIZE_MAX ? UINT64_MAX : (uint64_t)max_terms;
        return t;
    }
};

// One Pauli string in the reference's text format (PauliStringUtils.h:41-98):
// [+|-][i]<ops>, qubit q is character q, I/X/Y/Z.
struct ParsedString {
    std::vector<uint64_t> x, z;
    uint8_t flags = 0;
    std::size_t num_qubits = 0;
};

inline ParsedString parse_pauli(const std::string& s, std::size_t words) {
    if (s.empty()) throw std::invalid_argument("Pauli string is empty");
    ParsedString p;
    std::size_t pos = 0;
    bool sign = false, imag = false;
    if (s.compare(0, 2, "-i") == 0) {
        sign = imag = true;
        pos = 2;
    } else if (s.compare(0, 2, "+i") == 0) {
        imag = true;
        pos = 2;
    } else if (s[0] == '-') {
        sign = true;
        pos = 1;
    } else if (s[0] == '+' || s[0] == 'i') {
        imag = s[0] == 'i';
        pos = 1;
    }
    p.num_qubits = s.size() - pos;
    if (p.num_qubits > 64 * words) throw std::invalid_argument("Pauli string exceeds capacity");
    p.x.assign(words, 0);
    p.z.assign(words, 0);
    for (std::size_t q = 0; q < p.num_qubits; ++q) {
        const uint64_t bit = 1ull << (q % 64);
        switch (s[pos + q]) {
            case 'I': break;
            case 'X': p.x[q / 64] |= bit; break;
            case 'Z': p.z[q / 64] |= bit; break;
            case 'Y': p.x[q / 64] |= bit; p.z[q / 64] |= bit; break;
            default: throw std::invalid_argument("Invalid Pauli character");
        }
    }
    p.flags = (uint8_t)((sign ? 2 : 0) | (imag ? 1 : 0));
    return p;
}

template <std::size_t N, typename T = double>
class PauliSum {
    static_assert(std::is_same<T, double>::value, "device sums hold FP64 coefficients");

public:
    static constexpr std::size_t ArraySize = (N + 63) / 64;
    static_assert(ArraySize >= 1 && ArraySize <= PL_MAX_ARRAY_SIZE, "N out of range");

    // Host mirror of the device planes (download() / upload()).
    std::vector<std::vector<uint64_t>> x_data, z_data;
    std::vector<uint8_t> flags;
    std::vector<T> value;

    explicit PauliSum(std::size_t num_qubits = N, cudaStream_t stream = nullptr)
        : nq_(num_qubits), st_(stream) {
        if (num_qubits > N) throw std::invalid_argument("qubit count exceeds capacity");
        check(pl_state_create(&s_, (int)ArraySize, 1 << 16, st_), "PauliSum");
        clear_mirror();
    }
    PauliSum(const std::vector<std::pair<std::string, T>>& terms, cudaStream_t stream = nullptr)
        : PauliSum(N, stream) {
        std::size_t nq = 0;
        for (const auto& t : terms) {
            const ParsedString p = parse_pauli(t.first, ArraySize);
            for (std::size_t k = 0; k < ArraySize; ++k) {
                x_data[k].push_back(p.x[k]);
                z_data[k].push_back(p.z[k]);
            }
            flags.push_back(p.flags);
            value.push_back(t.second);
            if (p.num_qubits > nq) nq = p.num_qubits;
        }
        nq_ = terms.empty() ? N : nq;
        upload();
    }
    explicit PauliSum(const std::vector<std::string>& strings, cudaStream_t stream = nullptr)
        : PauliSum(with_unit(strings), stream) {}
    PauliSum(std::size_t num_qubits, const std::string& s, T c, cudaStream_t stream = nullptr)
        : PauliSum(std::vector<std::pair<std::string, T>>{{s, c}}, stream) {
        nq_ = num_qubits;
    }

    PauliSum(const PauliSum& o) : PauliSum(o.nq_, o.st_) {
        PauliSum& src = const_cast<PauliSum&>(o);
        check(pl_state_append(s_, src.s_), "PauliSum copy");
    }
    PauliSum& operator=(const PauliSum& o) {
        if (this != &o) {
            PauliSum tmp(o);
            swap(tmp);
        }
        return *this;
    }
    PauliSum(PauliSum&& o) noexcept { swap(o); }
    PauliSum& operator=(PauliSum&& o) noexcept {
        swap(o);
        return *this;
    }
    ~PauliSum() {
        if (s_) pl_state_destroy(s_);
    }
    void swap(PauliSum& o) noexcept {
        std::swap(s_, o.s_);
        std::swap(nq_, o.nq_);
        std::swap(st_, o.st_);
        x_data.swap(o.x_data);
        z_data.swap(o.z_data);
        flags.swap(o.flags);
        value.swap(o.value);
    }

    std::size_t num_qubits() const { return nq_; }
    std::size_t get_length() const {
        int64_t n = 0;
        check(pl_state_size(s_, &n), "get_length");
        return (std::size_t)n;
    }
    pl_state* handle() const { return s_; }

    // Host mirror -> device (replaces the device sum).
    void upload() {
        const std::size_t n = value.size();
        std::vector<uint64_t> x(ArraySize * n), z(ArraySize * n);
        for (std::size_t k = 0; k < ArraySize; ++k)
            for (std::size_t i = 0; i < n; ++i) {
                x[k * n + i] = x_data[k][i];
                z[k * n + i] = z_data[k][i];
            }
        check(pl_state_upload(s_, x.data(), z.data(), flags.data(), value.data(), (int64_t)n),
              "upload");
    }
    // Device -> host mirror.
    void download() {
        int64_t n = 0;
        check(pl_state_download(s_, nullptr, nullptr, nullptr, nullptr, 0, &n), "download");
        std::vector<uint64_t> x(ArraySize * (std::size_t)n), z(ArraySize * (std::size_t)n);
        flags.assign((std::size_t)n, 0);
        value.assign((std::size_t)n, 0.0);
        if (n > 0)
            check(pl_state_download(s_, x.data(), z.data(), flags.data(), value.data(), n, &n),
                  "download");
        for (std::size_t k = 0; k < ArraySize; ++k) {
            x_data[k].assign(x.begin() + k * n, x.begin() + (k + 1) * n);
            z_data[k].assign(z.begin() + k * n, z.begin() + (k + 1) * n);
        }
    }

    // PauliSumOperations.h:369-461, PauliSumUtils.h:315-393.
    void sort_and_combine() { check(pl_state_sort_and_combine(s_), "sort_and_combine"); }
    void canonicalize() { check(pl_state_canonicalize(s_), "canonicalize"); }
    void cutoff(T eps) { check(pl_state_cutoff(s_, (double)eps), "cutoff"); }
    void truncate_weight(std::size_t w) {
        check(pl_state_truncate_weight(s_, (uint64_t)w), "truncate_weight");
    }
    void trim(std::size_t max_terms) { check(pl_state_trim(s_, (uint64_t)max_terms), "trim"); }
    void trim(std::size_t max_terms, const PauliSum& keep) {
        check(pl_state_trim_protected(s_, (uint64_t)max_terms, keep.s_), "trim");
    }
    // PauliSumOperations.h:256-306: this := this * rhs, result[i*n + j] =
    // this[j] * rhs[i].
    void multiply(const PauliSum& rhs) { check(pl_state_multiply(s_, rhs.s_), "multiply"); }
    PauliSum& operator*=(const PauliSum& rhs) {
        multiply(rhs);
        return *this;
    }
    PauliSum operator*(const PauliSum& rhs) const {
        PauliSum out(*this);
        out.multiply(rhs);
        return out;
    }
    // PauliSumCore.h:210-237: append, then sort_and_combine.
    PauliSum& operator+=(const PauliSum& rhs) {
        check(pl_state_append(s_, rhs.s_), "operator+=");
        sort_and_combine();
        return *this;
    }
    PauliSum operator+(const PauliSum& rhs) const {
        PauliSum out(*this);
        out += rhs;
        return out;
    }
    // PauliSumOperations.h:107-183: each rotation (generator P = term,
    // angle = coefficient) in order, each followed by the `+=` merge.
    void evolve(const PauliSum& rotations) {
        PauliSum& r = const_cast<PauliSum&>(rotations);
        r.download();
        const std::size_t n = r.value.size();
        std::vector<uint64_t> x(ArraySize * n), z(ArraySize * n);
        for (std::size_t k = 0; k < ArraySize; ++k)
            for (std::size_t i = 0; i < n; ++i) {
                x[k * n + i] = r.x_data[k][i];
                z[k * n + i] = r.z_data[k][i];
            }
        check(pl_state_evolve(s_, x.data(), z.data(), r.flags.data(), r.value.data(),
                              (int64_t)n),
              "evolve");
    }
    // PauliSumClifford.h:213-239.
    void apply_CNOT(std::size_t control, std::size_t target) {
        check(pl_state_apply_cnot(s_, (int)control, (int)target), "apply_CNOT");
    }
    // Bulk Clifford gates (PauliSumClifford.h:44-501).
    void apply_H(std::size_t q) { gate1(PL_GATE_H, q); }
    void apply_S(std::size_t q) { gate1(PL_GATE_S, q); }
    void apply_H_YZ(std::size_t q) { gate1(PL_GATE_H_YZ, q); }
    void apply_H_XY(std::size_t q) { gate1(PL_GATE_H_XY, q); }
    void apply_sqrt_X(std::size_t q) { gate1(PL_GATE_SQRT_X, q); }
    void apply_sqrt_Y(std::size_t q) { gate1(PL_GATE_SQRT_Y, q); }
    void apply_X(std::size_t q) { gate1(PL_GATE_X, q); }
    void apply_Y(std::size_t q) { gate1(PL_GATE_Y, q); }
    void apply_Z(std::size_t q) { gate1(PL_GATE_Z, q); }
    void apply_I(std::size_t q) { gate1(PL_GATE_I, q); }
    void apply_CZ(std::size_t c, std::size_t t) { gate2(PL_GATE_CZ, c, t); }
    void apply_CY(std::size_t c, std::size_t t) { gate2(PL_GATE_CY, c, t); }
    void apply_XC_X(std::size_t c, std::size_t t) { gate2(PL_GATE_XC_X, c, t); }
    void apply_XC_Y(std::size_t c, std::size_t t) { gate2(PL_GATE_XC_Y, c, t); }
    void apply_XC_Z(std::size_t c, std::size_t t) { gate2(PL_GATE_XC_Z, c, t); }
    void apply_YC_X(std::size_t c, std::size_t t) { gate2(PL_GATE_YC_X, c, t); }
    void apply_YC_Y(std::size_t c, std::size_t t) { gate2(PL_GATE_YC_Y, c, t); }
    void apply_YC_Z(std::size_t c, std::size_t t) { gate2(PL_GATE_YC_Z, c, t); }
    void apply_SWAP(std::size_t a, std::size_t b) { gate2(PL_GATE_SWAP, a, b); }
    void apply_iSWAP(std::size_t a, std::size_t b) { gate2(PL_GATE_ISWAP, a, b); }
    // apply_RX / RY / RZ (PauliSumOperations.h:29-104): exp(-i angle/2 P).
    void apply_RX(std::size_t q, T angle) { rgate(1, q, angle); }
    void apply_RY(std::size_t q, T angle) { rgate(2, q, angle); }
    void apply_RZ(std::size_t q, T angle) { rgate(3, q, angle); }

    // PauliSumUtils.h:163-177.
    T zero_state_expectation() const {
        double r = 0.0;
        check(pl_state_zero_state_expectation(s_, &r), "zero_state_expectation");
        return r;
    }
    // PauliSumUtils.h:178-268, 400-410.
    T basis_state_expectation(const std::string& bits) const {
        if (bits.size() != nq_)
            throw std::invalid_argument("basis_state_expectation: bit string length " +
                                        std::to_string(bits.size()) + " does not match " +
                                        std::to_string(nq_) + " qubits");
        std::vector<uint64_t> w(ArraySize, 0);
        for (std::size_t q = 0; q < bits.size(); ++q) {
            if (bits[q] != '0' && bits[q] != '1')
                throw std::invalid_argument(
                    "basis_state_expectation: bit string must contain only '0'/'1'");
            if (bits[q] == '1') w[q / 64] |= 1ull << (q % 64);
        }
        double r = 0.0;
        check(pl_state_basis_state_expectation(s_, w.data(), &r), "basis_state_expectation");
        return r;
    }
    T trace() const {
        double r = 0.0;
        check(pl_state_trace(s_, (int)nq_, &r), "trace");
        return r;
    }
    T frobenius_norm2() const {
        double r = 0.0;
        check(pl_state_frobenius_norm2(s_, &r), "frobenius_norm2");
        return r;
    }
    T lookup(const std::string& pauli_string) const {
        const ParsedString p = parse_pauli(pauli_string, ArraySize);
        double r = 0.0;
        check(pl_state_lookup(s_, p.x.data(), p.z.data(), p.flags, &r), "lookup");
        return r;
    }

    // PauliSumUtils.h:19-33: "%f * <string>" per term.
    std::string get_str() {
        download();
        static const char* pre[4] = {"", "i", "-", "-i"};
        std::string out;
        char buf[64];
        for (std::size_t i = 0; i < value.size(); ++i) {
            std::snprintf(buf, sizeof(buf), "%f * ", value[i]);
            out += buf;
            out += pre[flags[i] & 3];
            for (std::size_t q = 0; q < nq_; ++q) {
                const bool xb = (x_data[q / 64][i] >> (q % 64)) & 1u;
                const bool zb = (z_data[q / 64][i] >> (q % 64)) & 1u;
                out += xb && zb ? 'Y' : xb ? 'X' : zb ? 'Z' : 'I';
            }
            out += '\n';
        }
        return out;
    }

private:
    void gate1(int g, std::size_t q) {
        check(pl_state_apply_clifford(s_, g, (int)q, (int)q), "apply gate");
    }
    void gate2(int g, std::size_t a, std::size_t b) {
        check(pl_state_apply_clifford(s_, g, (int)a, (int)b), "apply gate");
    }
    void rgate(int axis, std::size_t q, T angle) {
        check(pl_state_apply_rotation_gate(s_, axis, (int)q, (double)angle), "apply rotation");
    }
    static std::vector<std::pair<std::string, T>> with_unit(const std::vector<std::string>& v) {
        std::vector<std::pair<std::string, T>> out;
        for (const auto& s : v) out.emplace_back(s, T(1));
        return out;
    }
    void clear_mirror() {
        x_data.assign(ArraySize, {});
        z_data.assign(ArraySize, {});
        flags.clear();
        value.clear();
    }

    pl_state* s_ = nullptr;
    std::size_t nq_ = N;
    cudaStream_t st_ = nullptr;
};

// [A, B] and i[A, B], uncombined, in the reference's single-threaded order
// (PauliSumOperations.h:316-356).
template <std::size_t N, typename T>
PauliSum<N, T> commutator(const PauliSum<N, T>& a, const PauliSum<N, T>& b) {
    PauliSum<N, T> out(a.num_qubits());
    check(pl_state_commutator(out.handle(), a.handle(), b.handle(), 0), "commutator");
    return out;
}
template <std::size_t N, typename T>
PauliSum<N, T> i_commutator(const PauliSum<N, T>& a, const PauliSum<N, T>& b) {
    PauliSum<N, T> out(a.num_qubits());
    check(pl_state_commutator(out.handle(), a.handle(), b.handle(), 1), "i_commutator");
    return out;
}

// trace_product (PauliSumUtils.h:412-447): Re tr(A B).
template <std::size_t N, typename T>
T trace_product(const PauliSum<N, T>& a, const PauliSum<N, T>& b) {
    if (a.num_qubits() != b.num_qubits())
        throw std::invalid_argument("trace_product: qubit-count mismatch");
    double r = 0.0;
    check(pl_state_trace_product(a.handle(), b.handle(), (int)a.num_qubits(), &r),
          "trace_product");
    return r;
}

// propagate (PauliPropagation.h:54-63): the rotations (generator = term,
// angle = coefficient) in reverse order, each evolve + apply_truncation.
template <std::size_t N, typename T>
PauliSum<N, T> propagate(const PauliSum<N, T>& observable, const PauliSum<N, T>& rotations,
                         const TruncationOptions<T>& opts = TruncationOptions<T>{}) {
    PauliSum<N, T> out(observable);
    PauliSum<N, T>& r = const_cast<PauliSum<N, T>&>(rotations);
    r.download();
    const std::size_t n = r.value.size();
    constexpr std::size_t AS = PauliSum<N, T>::ArraySize;
    std::vector<uint64_t> x(AS * n), z(AS * n);
    for (std::size_t k = 0; k < AS; ++k)
        for (std::size_t i = 0; i < n; ++i) {
            x[k * n + i] = r.x_data[k][i];
            z[k * n + i] = r.z_data[k][i];
        }
    const pl_truncation t = opts.c_abi();
    check(pl_propagate(out.handle(), x.data(), z.data(), r.flags.data(), r.value.data(),
                       (int64_t)n, nullptr, 0, &t),
          "propagate");
    return out;
}

// propagate_expectation (PauliPropagation.h:65-71): <0|U^dagger O U|0>.
template <std::size_t N, typename T>
T propagate_expectation(const PauliSum<N, T>& observable, const PauliSum<N, T>& rotations,
                        const TruncationOptions<T>& opts = TruncationOptions<T>{}) {
    return propagate(observable, rotations, opts).zero_state_expectation();
}

}  // namespace paulib_b200
