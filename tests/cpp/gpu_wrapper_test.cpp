// The reference's own GPU host wrapper, include/gpu/GpuPauliSum.h
// (GpuPauliSum, gpu_multiply, gpu_commutator: :35-238), compiled unchanged
// against libpaulib_b200.so, which supplies the two launchers the wrapper
// calls (launch_gpu_mul_soa, launch_gpu_commutator_soa).  The results are
// checked against the reference's own CPU code on the same random sums:
// the product term by term in its i*n + j order, the commutators term by
// term against the single-threaded CPU commutator (the deterministic order
// this library emits in).  Prints "<passed> passed, <failed> failed".
#include <cstdio>

#include <omp.h>

#include "PauliSum.h"
#include "gpu/GpuPauliSum.h"

static int g_pass = 0, g_fail = 0;

template <std::size_t N>
static void expect_same(const char* what, const paulib::PauliSum<N, double>& got,
                        const paulib::PauliSum<N, double>& want) {
    bool ok = got.get_length() == want.get_length() && got.flags == want.flags &&
              got.value == want.value;
    for (std::size_t k = 0; ok && k < paulib::PauliSum<N, double>::ArraySize; ++k)
        ok = got.x_data[k] == want.x_data[k] && got.z_data[k] == want.z_data[k];
    if (ok) {
        ++g_pass;
    } else {
        ++g_fail;
        std::printf("FAIL %s: %zu vs %zu terms\n", what, got.get_length(), want.get_length());
    }
}

template <std::size_t N>
static void run(std::size_t nq, std::size_t n, std::size_t m) {
    using PS = paulib::PauliSum<N, double>;
    const PS a = paulib::random_pauli_sum<N, double>(n, 11, nq);
    const PS b = paulib::random_pauli_sum<N, double>(m, 12, nq);
    paulib::GpuPauliSum<N> ga(a), gb(b);
    PS cpu = a;
    cpu.multiply(b);
    expect_same("gpu_multiply", paulib::gpu_multiply(ga, gb).download(), cpu);
    const int threads = omp_get_max_threads();
    omp_set_num_threads(1);
    const PS c = paulib::commutator(a, b), ic = paulib::i_commutator(a, b);
    omp_set_num_threads(threads);
    expect_same("gpu_commutator", paulib::gpu_commutator(ga, gb).download(), c);
    expect_same("gpu_commutator(i)", paulib::gpu_commutator(ga, gb, true).download(), ic);
}

int main() {
    try {
        run<64>(40, 300, 200);
        run<128>(100, 120, 90);
        run<256>(256, 64, 50);
    } catch (const std::exception& e) {
        std::printf("FAIL exception: %s\n", e.what());
        ++g_fail;
    }
    std::printf("%d passed, %d failed\n", g_pass, g_fail);
    return g_fail ? 1 : 0;
}
