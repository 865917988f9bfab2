/*
 * paulib_b200.h -- C ABI of the B200 Pauli-sum library (libpaulib_b200.so).
 *
 * Plain pointers and sizes only; includable from C, C++ (g++) and nvcc
 * translation units, like the reference seam include/gpu/paulib_gpu_api.h
 * (:1-14).  A Pauli sum crosses the boundary as SoA planes:
 *
 *   x[k*stride + i], z[k*stride + i]   word k of term i (I=00, X=10, Z=01,
 *                                       Y=11 in (x,z) bits)
 *   flags[i]                            exponent of i^k: bit0 imaginary,
 *                                       bit1 sign
 *   val[i]                              FP64 coefficient
 *
 * where stride is the plane length (n for inputs, the stated capacity for
 * outputs).  array_size = ceil(N/64) words per string, 1..16.
 *
 * Every pl_* entry point returns a status code (PL_OK on success) and never
 * traps or aborts; the two launch_gpu_* drop-ins keep the reference's void
 * signature and record their status for pl_get_last_error().
 */
#ifndef PAULIB_B200_H
#define PAULIB_B200_H

#include <stddef.h>
#include <stdint.h>

#include <cuda_runtime_api.h>

#if defined(__GNUC__)
#define PL_API __attribute__((visibility("default")))
#else
#define PL_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PL_OK 0
#define PL_ERR_INVALID_ARG 1   /* bad size, array_size, pointer or option   */
#define PL_ERR_OOM 2           /* device allocation failed                  */
#define PL_ERR_TIMEOUT 3       /* a bounded device-side wait ran out        */
#define PL_ERR_CUDA 4          /* a CUDA runtime call failed                */
#define PL_ERR_CAPACITY 5      /* output would exceed the stated capacity   */
#define PL_ERR_UNSUPPORTED 6   /* valid request outside what is built       */
#define PL_ERR_INTERNAL 7      /* device-side consistency check failed      */
#define PL_ERR_CANCELLED 8     /* the caller's cancel flag stopped the work */

#define PL_MAX_ARRAY_SIZE 16

PL_API const char* pl_status_string(int status);
/* Status of the most recent call on the calling host thread (the void
 * drop-ins report through this). */
PL_API int pl_get_last_error(void);
PL_API const char* pl_last_error_message(void);
PL_API int pl_version(void);

/* ---- product and commutator ------------------------------------------- */

/* Drop-in for launch_gpu_mul_soa (include/gpu/paulib_gpu_api.h:25-33):
 * out[i*n + j] = lhs[j] * rhs[i] for j < n, i < m; out planes have stride
 * n*m.  Device pointers, asynchronous on `stream`.  An unsupported
 * array_size records PL_ERR_INVALID_ARG instead of trapping. */
PL_API void launch_gpu_mul_soa(int array_size, const uint64_t* lhs_x, const uint64_t* lhs_z,
                        const uint8_t* lhs_flags, const double* lhs_val,
                        const uint64_t* rhs_x, const uint64_t* rhs_z,
                        const uint8_t* rhs_flags, const double* rhs_val, uint64_t* out_x,
                        uint64_t* out_z, uint8_t* out_flags, double* out_val, int n, int m,
                        cudaStream_t stream);

/* Drop-in for launch_gpu_commutator_soa (include/gpu/paulib_gpu_api.h:43-53):
 * [lhs, rhs] (multiply_by_i = 0) or i[lhs, rhs] (= 1).  Anticommuting pairs
 * emit lhs_j * rhs_i with value 2*lhs_val[j]*rhs_val[i] into planes of
 * stride `capacity`, starting at slot *d_count (zeroed by the caller, as in
 * the reference); *d_count ends at the number of emitted terms.  Unlike the
 * reference's atomic slot claim, the emission order is deterministic:
 * lhs-major, rhs-minor, the order of the reference's single-threaded CPU
 * commutator_impl (PauliSumOperations.h:316-346).  Asynchronous on `stream`,
 * like the reference's launcher: the host never waits, and the look-back
 * scratch is allocated and released in stream order.  Terms beyond
 * `capacity` are not written (the reference writes past the end); *d_count
 * still ends at the full count, so *d_count > capacity after the stream
 * completes means the output did not fit. */
PL_API void launch_gpu_commutator_soa(int array_size, int multiply_by_i, const uint64_t* lhs_x,
                               const uint64_t* lhs_z, const uint8_t* lhs_flags,
                               const double* lhs_val, const uint64_t* rhs_x,
                               const uint64_t* rhs_z, const uint8_t* rhs_flags,
                               const double* rhs_val, uint64_t* out_x, uint64_t* out_z,
                               uint8_t* out_flags, double* out_val,
                               unsigned long long* d_count, int n, int m, long long capacity,
                               cudaStream_t stream);

/* Status-returning form of launch_gpu_mul_soa with 64-bit sizes
 * (n*m < 2^40).  Replaces the same reference interface. */
PL_API int pl_multiply(int array_size, const uint64_t* lhs_x, const uint64_t* lhs_z,
                const uint8_t* lhs_flags, const double* lhs_val, int64_t n,
                const uint64_t* rhs_x, const uint64_t* rhs_z, const uint8_t* rhs_flags,
                const double* rhs_val, int64_t m, uint64_t* out_x, uint64_t* out_z,
                uint8_t* out_flags, double* out_val, cudaStream_t stream);

/* Status-returning form of launch_gpu_commutator_soa (same semantics and
 * deterministic order); the pair count n*m must be below 2^40. */
PL_API int pl_commutator(int array_size, int multiply_by_i, const uint64_t* lhs_x,
                  const uint64_t* lhs_z, const uint8_t* lhs_flags, const double* lhs_val,
                  int64_t n, const uint64_t* rhs_x, const uint64_t* rhs_z,
                  const uint8_t* rhs_flags, const double* rhs_val, int64_t m, uint64_t* out_x,
                  uint64_t* out_z, uint8_t* out_flags, double* out_val, int64_t capacity,
                  unsigned long long* d_count, cudaStream_t stream);

/* pl_commutator for callers that cannot let the library allocate device
 * memory -- hosts that own the whole device through their own pool or an
 * HBM budget, and callers that cannot afford the synchronisation an
 * allocation may cause.  No counterpart in the reference.  Same arguments,
 * result and order as pl_commutator; its scratch is a static 512 KB device
 * array of this library, so n*m is limited to 2^29 pairs (larger requests
 * return PL_ERR_INVALID_ARG).  The first call on a device looks the array's
 * address up (cudaGetSymbolAddress); make that first call before any stream
 * capture.  All calls share the array: calls that overlap on the GPU (other
 * streams, other threads) race and must be serialised by the caller.
 * Synchronous, like pl_commutator: before it returns it waits for the
 * stream, because it copies the 4-byte device status back to the host.
 * Calls no cudaMalloc / cudaFree / cudaHostAlloc. */
PL_API int pl_commutator_noalloc(int array_size, int multiply_by_i, const uint64_t* lhs_x,
                                 const uint64_t* lhs_z, const uint8_t* lhs_flags,
                                 const double* lhs_val, int64_t n, const uint64_t* rhs_x,
                                 const uint64_t* rhs_z, const uint8_t* rhs_flags,
                                 const double* rhs_val, int64_t m, uint64_t* out_x,
                                 uint64_t* out_z, uint8_t* out_flags, double* out_val,
                                 int64_t capacity, unsigned long long* d_count,
                                 cudaStream_t stream);

/* ---- collate: sort_and_combine / canonicalize / cutoff / weight ------- */

/* canonicalize() (PauliSumUtils.h:315-328): fold the sign bit into the
 * value, merge equal (x, z, phase), drop exact zeros.  Output sorted by
 * (x[0..AS), z[0..AS), phase). */
#define PL_COLLATE_CANONICALIZE 0
/* sort_and_combine() (PauliSumOperations.h:369-461): key (x, z, flags)
 * with the sign kept in the key; zero sums are kept. */
#define PL_COLLATE_SORT_AND_COMBINE 1

typedef struct {
    int32_t mode;          /* PL_COLLATE_* */
    int32_t reserved;
    double cutoff;         /* > 0: then drop |c| < cutoff (cutoff(),
                              PauliSumUtils.h:378-384) */
    uint64_t max_weight;   /* != UINT64_MAX: then drop weight > max_weight
                              (truncate_weight(), PauliSumUtils.h:387-393) */
} pl_collate_opts;

/* Workspace needed to collate n input terms. */
PL_API int pl_collate_workspace_size(int array_size, int64_t n, size_t* bytes);

/* Collate n terms (planes of stride n) into out planes of stride
 * out_capacity.  Synchronous: returns after `stream` drained, with the
 * output term count in *out_count (host pointer).  Within an output
 * segment coefficients are summed in input-index order (segments longer
 * than 32 terms use a fixed-order parallel reduction).  n < 2^30.
 * Replaces PauliSum::canonicalize / sort_and_combine / cutoff /
 * truncate_weight (PauliSumUtils.h:287-393, PauliSumOperations.h:369-461). */
PL_API int pl_collate(int array_size, const uint64_t* x, const uint64_t* z, const uint8_t* flags,
               const double* val, int64_t n, uint64_t* out_x, uint64_t* out_z,
               uint8_t* out_flags, double* out_val, int64_t out_capacity, int64_t* out_count,
               const pl_collate_opts* opts, void* workspace, size_t workspace_bytes,
               cudaStream_t stream);

/* Workspace needed by pl_multiply_collate for n x m products. */
PL_API int pl_multiply_collate_workspace_size(int array_size, int64_t n, int64_t m, size_t* bytes);

/* Fused `a *= b; a.canonicalize()` (PauliSumOperations.h:256-306 then
 * PauliSumUtils.h:315-328): the n*m products (in the reference's i*n + j
 * order) are generated inside the sort and never written to HBM.  Output
 * and synchronisation as pl_collate.  n*m < 2^30. */
PL_API int pl_multiply_collate(int array_size, const uint64_t* lhs_x, const uint64_t* lhs_z,
                        const uint8_t* lhs_flags, const double* lhs_val, int64_t n,
                        const uint64_t* rhs_x, const uint64_t* rhs_z,
                        const uint8_t* rhs_flags, const double* rhs_val, int64_t m,
                        uint64_t* out_x, uint64_t* out_z, uint8_t* out_flags, double* out_val,
                        int64_t out_capacity, int64_t* out_count, const pl_collate_opts* opts,
                        void* workspace, size_t workspace_bytes, cudaStream_t stream);

/* ---- single-pass term kernels ----------------------------------------- */

/* apply_CNOT(c, t) in place (PauliSumClifford.h:213-239); order kept. */
PL_API int pl_apply_cnot(int array_size, uint64_t* x, uint64_t* z, uint8_t* flags, int64_t n,
                  int64_t stride, int control, int target, cudaStream_t stream);

/* zero_state_expectation (PauliSumUtils.h:163-177) into *d_result (device
 * double).  Fixed-order reduction, so run-to-run deterministic. */
PL_API int pl_zero_state_expectation(int array_size, const uint64_t* x, const uint8_t* flags,
                              const double* val, int64_t n, int64_t stride, double* d_result,
                              cudaStream_t stream);

/* ---- device-resident propagation state -------------------------------- */

/* TruncationOptions<double> (PauliPropagation.h:27-31). */
typedef struct {
    uint64_t max_weight;          /* UINT64_MAX = disabled */
    double coefficient_cutoff;    /* <= 0 = disabled */
    uint64_t max_terms;           /* UINT64_MAX = disabled */
} pl_truncation;

/* Bulk Clifford gates (PauliSumClifford.h:44-501).  One-qubit gates act on
 * qubit a; two-qubit gates on control / first qubit a and target / second
 * qubit b (a != b). */
#define PL_GATE_H 1
#define PL_GATE_S 2
#define PL_GATE_H_YZ 3
#define PL_GATE_H_XY 4
#define PL_GATE_SQRT_X 5
#define PL_GATE_SQRT_Y 6
#define PL_GATE_X 7
#define PL_GATE_Y 8
#define PL_GATE_Z 9
#define PL_GATE_I 10
#define PL_GATE_CNOT 11
#define PL_GATE_CZ 12
#define PL_GATE_CY 13
#define PL_GATE_XC_X 14
#define PL_GATE_XC_Y 15
#define PL_GATE_XC_Z 16
#define PL_GATE_YC_X 17
#define PL_GATE_YC_Y 18
#define PL_GATE_YC_Z 19
#define PL_GATE_SWAP 20
#define PL_GATE_ISWAP 21

/* Circuit ops, rows of int32 (kind, a, b) in application order. */
#define PL_OP_ROTATION 0   /* rotation number a of the rotation table */
#define PL_OP_CNOT 1       /* CNOT control a, target b */
#define PL_OP_CLIFFORD 100 /* kind PL_OP_CLIFFORD + g: Clifford gate PL_GATE_g on a (, b) */

typedef struct pl_state pl_state;

/* A Pauli sum kept in device memory between gates.  capacity_hint sizes
 * the initial buffers (terms); the state grows on demand. */
PL_API int pl_state_create(pl_state** state, int array_size, int64_t capacity_hint,
                    cudaStream_t stream);
PL_API int pl_state_destroy(pl_state* state);
/* Host planes (stride n) -> device. */
PL_API int pl_state_upload(pl_state* state, const uint64_t* x, const uint64_t* z,
                    const uint8_t* flags, const double* val, int64_t n);
/* Device -> host planes of stride *n (call with x == NULL to query n). */
PL_API int pl_state_download(pl_state* state, uint64_t* x, uint64_t* z, uint8_t* flags,
                      double* val, int64_t capacity, int64_t* n);
PL_API int pl_state_size(pl_state* state, int64_t* n);

/* PauliSum::evolve(rotations) (PauliSumOperations.h:107-183): the n_rot
 * rotations (host planes, stride n_rot; val = angle) applied in order,
 * each followed by the reference's `+=` merge only. */
PL_API int pl_state_evolve(pl_state* state, const uint64_t* rot_x, const uint64_t* rot_z,
                    const uint8_t* rot_flags, const double* rot_theta, int64_t n_rot);
/* apply_truncation (PauliPropagation.h:36-47). */
PL_API int pl_state_apply_truncation(pl_state* state, const pl_truncation* opts);
PL_API int pl_state_canonicalize(pl_state* state);
PL_API int pl_state_sort_and_combine(pl_state* state);
PL_API int pl_state_cutoff(pl_state* state, double eps);
PL_API int pl_state_truncate_weight(pl_state* state, uint64_t max_weight);
PL_API int pl_state_apply_cnot(pl_state* state, int control, int target);
/* apply_H, apply_S, ..., apply_iSWAP (PauliSumClifford.h:44-501): gate
 * PL_GATE_* on qubit q1 (and q2 for two-qubit gates), every term in place. */
PL_API int pl_state_apply_clifford(pl_state* state, int gate, int q1, int q2);
/* apply_RX / apply_RY / apply_RZ (PauliSumOperations.h:29-104): the gate
 * exp(-i angle/2 P) on `qubit`, P = X (axis 1), Y (2) or Z (3), followed by
 * the reference's `+=` merge (sort_and_combine). */
PL_API int pl_state_apply_rotation_gate(pl_state* state, int axis, int qubit, double angle);
/* trim(max_terms) (PauliSumUtils.h:331-345): keep the max_terms terms of
 * largest |c| in their order; among equal |c| at the boundary the lower
 * index survives (the reference leaves that choice to std::nth_element). */
PL_API int pl_state_trim(pl_state* state, uint64_t max_terms);
/* trim(max_terms, keep) (PauliSumUtils.h:347-375): terms whose (x, z)
 * pattern occurs in `keep` are always kept and the others share what is
 * left of max_terms. */
PL_API int pl_state_trim_protected(pl_state* state, uint64_t max_terms, pl_state* keep);
PL_API int pl_state_zero_state_expectation(pl_state* state, double* result);
/* basis_state_expectation (PauliSumUtils.h:178-220): <x| sum |x> for the
 * basis state whose bit q (word q/64, bit q%64 of bit_words[0..AS)) is
 * qubit q's value. */
PL_API int pl_state_basis_state_expectation(pl_state* state, const uint64_t* bit_words,
                                            double* result);
/* trace (PauliSumUtils.h:226-245): 2^num_qubits times the signed sum of the
 * real-phase identity terms. */
PL_API int pl_state_trace(pl_state* state, int num_qubits, double* result);
/* frobenius_norm2 (PauliSumUtils.h:400-410): sum of squared coefficients
 * (tr(O^dagger O) / 2^n of a canonical sum). */
PL_API int pl_state_frobenius_norm2(pl_state* state, double* result);
/* lookup (PauliSumUtils.h:246-268): coefficient of the string (x, z words,
 * flags), phases relative to the query, +-i terms skipped. */
PL_API int pl_state_lookup(pl_state* state, const uint64_t* x, const uint64_t* z,
                           uint8_t flags, double* result);
/* trace_product (PauliSumUtils.h:412-447): Re tr(A B) = 2^num_qubits times the
 * sum over shared patterns of Re(w_A * w_B). */
PL_API int pl_state_trace_product(pl_state* a, pl_state* b, int num_qubits, double* result);

/* lhs := lhs * rhs, the outer product in the reference's i*n + j order
 * (PauliSum::multiply, PauliSumOperations.h:256-306).  lhs and rhs may be
 * the same state. */
PL_API int pl_state_multiply(pl_state* lhs, pl_state* rhs);
/* lhs := canonicalize(lhs * rhs) without materialising the products
 * (`a *= b; a.canonicalize()`). */
PL_API int pl_state_multiply_canonicalize(pl_state* lhs, pl_state* rhs);
/* out := [a, b] (multiply_by_i = 0) or i[a, b] (= 1), uncombined, in the
 * reference's single-threaded CPU order (commutator / i_commutator,
 * PauliSumOperations.h:316-356). */
PL_API int pl_state_commutator(pl_state* out, pl_state* a, pl_state* b, int multiply_by_i);
/* dst := dst followed by the terms of src (PauliSum::add, PauliSumCore.h:
 * 210-237, before its merge); the reference's `+=` is this followed by
 * pl_state_sort_and_combine. */
PL_API int pl_state_append(pl_state* dst, pl_state* src);

/* propagate (PauliPropagation.h:54-63): ops walked in reverse; a rotation
 * is evolve + apply_truncation, a CNOT is apply_CNOT.  ops == NULL means
 * "every rotation in order", the reference's rotation-only circuit. */
PL_API int pl_propagate(pl_state* state, const uint64_t* rot_x, const uint64_t* rot_z,
                 const uint8_t* rot_flags, const double* rot_theta, int64_t n_rot,
                 const int32_t* ops, int64_t n_ops, const pl_truncation* opts);

/* State options (pl_state_set_option). */
#define PL_OPT_GRAPHS 1  /* value != 0: runs of single-qubit rotations replay a captured
                            CUDA graph of their kernel chain (gate records live in device
                            memory, so one graph serves every run of that length) */
#define PL_OPT_GATE_LOG 2  /* value != 0: every fast-path rotation of pl_propagate records
                              its sizes (terms in, anticommuting terms, terms out) in a
                              device log, one i64 triple per op in processing order (the
                              circuit reversed); other ops record zeros.  For byte models;
                              no counterpart in the reference. */
PL_API int pl_state_set_option(pl_state* state, int option, int64_t value);
/* Cancellation: while `flag` (host memory, or NULL to clear) is non-zero,
 * pl_propagate stops between gates -- it drains the work already queued
 * and returns PL_ERR_CANCELLED, leaving the state holding the sum after
 * the last gate that ran. */
PL_API int pl_state_set_cancel_flag(pl_state* state, const int32_t* flag);
/* Copy the gate log of the state's last pl_propagate (PL_OPT_GATE_LOG):
 * min(max_ops, *n_ops) triples into sizes[3*q .. 3*q+2]; synchronous. */
PL_API int pl_state_gate_log(pl_state* state, int64_t* sizes, int64_t max_ops,
                             int64_t* n_ops);
/* Device bytes the state's buffers and workspace hold. */
PL_API int pl_state_memory(pl_state* state, uint64_t* bytes);

/* ---- sharded sums: hash-owned collate across ranks ---------------------
 *
 * MpiPauliSum::exchange_and_combine (MpiPauliSum.h:101-181): every term is
 * owned by rank FNV-1a(x, z) mod ranks (the phase is excluded, so P, -P and
 * iP meet on one rank).  pl_state_shard_pack writes the state's terms as
 * term-major records (x[0..AS), z[0..AS), flags, value bits: 2*AS+2 u64 words
 * each) into `records` (device memory, >= n records), grouped by owner in
 * term order, and the per-owner counts into counts[0..ranks); the caller
 * exchanges the buckets (one all-to-all, e.g. NCCL), and the receiver loads
 * what it got with pl_state_shard_unpack and canonicalizes.  ranks <= 64. */
PL_API int pl_state_shard_pack(pl_state* state, int ranks, uint64_t* records, int64_t capacity,
                               int64_t* counts);
PL_API int pl_state_shard_unpack(pl_state* state, const uint64_t* records, int64_t n);
/* For the global trim of a sharded sum (MpiPauliSum.h:187-210): the number
 * of terms with |c| >= threshold, and the largest |c| (0 for an empty sum). */
PL_API int pl_state_count_above(pl_state* state, double threshold, int64_t* count);
PL_API int pl_state_max_abs(pl_state* state, double* result);

/* ---- many propagations on one device: batch and serving ---------------
 *
 * A job is one propagate_expectation (PauliPropagation.h:65-71): the
 * observable is uploaded, propagated backwards through the circuit with
 * truncation after every rotation, and reduced to zero_state_expectation.
 * Jobs run on `lanes` device-resident states, each with its own stream and
 * host thread, so the kernels of different jobs overlap on the GPU and the
 * host-side waits of one job hide behind the work of others.  The buffers
 * of all lanes count against an HBM budget: a lane that must grow past it
 * waits for others to release memory.  Every job computes exactly what
 * pl_propagate computes on its own: results do not depend on the mix. */
typedef struct {
    int array_size;
    const uint64_t* obs_x;       /* host planes, stride obs_n */
    const uint64_t* obs_z;
    const uint8_t* obs_flags;
    const double* obs_val;
    int64_t obs_n;
    const uint64_t* rot_x;       /* host planes, stride n_rot; rot_theta = angles */
    const uint64_t* rot_z;
    const uint8_t* rot_flags;
    const double* rot_theta;
    int64_t n_rot;
    const int32_t* ops;          /* (kind, a, b) rows as for pl_propagate */
    int64_t n_ops;
    pl_truncation trunc;
    double arrival_s;            /* pl_serve: seconds after its start the job arrives */
    const int32_t* cancel;       /* host flag or NULL: once non-zero, the job stops between
                                    gates (or does not start) with PL_ERR_CANCELLED */
} pl_job;

typedef struct {
    double expectation;          /* zero_state_expectation of the propagated sum */
    int64_t final_terms;
    int status;                  /* PL_OK or the job's error */
    int lane;
    double start_s;              /* seconds from the call's start */
    double end_s;
} pl_job_result;

#define PL_ORDER_GIVEN 0
#define PL_ORDER_LONGEST_FIRST 1  /* by estimated cost (rotations x words), descending */

typedef struct {
    int lanes;                   /* concurrent jobs, >= 1 */
    int use_graphs;              /* PL_OPT_GRAPHS for every lane */
    int order;                   /* pl_batch_propagate only */
    uint64_t hbm_budget;         /* bytes all lanes may hold; 0 = 85% of free device memory */
    uint64_t keep_bytes;         /* a lane keeps at most this between jobs; 0 = budget / lanes */
    cudaStream_t sync_stream;    /* work queued here before the call completes first (or NULL) */
} pl_batch_opts;

typedef struct {
    double wall_s;
    uint64_t peak_bytes;         /* peak of the budgeted bytes */
    uint64_t budget_waits;       /* times a lane waited for memory (admission or growth) */
    uint64_t jobs_failed;        /* jobs that ended with a status other than PL_OK */
    uint64_t jobs_rejected;      /* jobs refused at admission (PL_ERR_OOM, never started) */
    uint64_t admission_waits;    /* jobs deferred at admission until memory freed up */
} pl_batch_stats;

/* Admission estimate of one job (host-only arithmetic, no device work):
 * *terms bounds the terms its canonical sum can hold after any truncation
 * step, the least of
 *   (a) the Frobenius bound 2 * (sum |c|)^2 / cutoff^2: conjugation by the
 *       circuit keeps ||O||_F, truncation only removes terms, and every kept
 *       term has |c| >= cutoff (x2 for the two phases of one string);
 *   (b) the weight bound 2 * sum_{k <= min(w, s)} C(s, k) 3^k over the s
 *       qubits of the observable's light cone (its support grown through the
 *       circuit's two-qubit gates, walked in Heisenberg order);
 * and *bytes = 20 * S * terms + 64 MiB: the five term buffers of a state
 * (S = 16*AS + 9 bytes per term) at up to twice the live terms before a
 * truncation and twice again after a capacity doubling, plus workspace.
 * Saturates at UINT64_MAX.  pl_serve and pl_batch_propagate reserve
 * min(bytes, budget / lanes) (at least a fresh state's size) when they
 * admit the job, and refuse a job whose fresh state alone exceeds the
 * budget. */
PL_API int pl_job_estimate(const pl_job* job, uint64_t* terms, uint64_t* bytes);

/* All jobs available at once. */
PL_API int pl_batch_propagate(const pl_job* jobs, int64_t count, const pl_batch_opts* opts,
                              pl_job_result* results, pl_batch_stats* stats);
/* Jobs arrive at their arrival_s; each free lane takes the earliest arrived
 * job (continuous batching).  Latency of job i = end_s - arrival_s. */
PL_API int pl_serve(const pl_job* jobs, int64_t count, const pl_batch_opts* opts,
                    pl_job_result* results, pl_batch_stats* stats);

/* ---- tuning ------------------------------------------------------------- */

/* Keys per thread of the collate engine's onesweep digit pass: 8, 12 or 16
 * (tiles of 2048, 3072 or 4096 keys); 0 (default): 12 for index-packed
 * keys, 8 for key + payload passes.  Process-wide. */
#define PL_TUNE_RADIX_ITEMS 1
/* canonicalize() of a sum (or of a product) whose varying x / z bits and
 * term index fit one 64-bit word sorts index-packed keys: 8 bytes per key
 * and digit pass, digits over the x / z bits only, the phase split in the
 * segment sums.  0 (default) or 1: used where it fits; -1: never (the
 * general key + payload sort).  Results are identical either way. */
#define PL_TUNE_INDEX_KEYS 2
/* canonicalize() / sort_and_combine() of a sum whose plain key needs more
 * than 16 digit passes: when every term's x and z bits lie in two
 * consecutive words and within 16 consecutive bits of each (strings on a
 * window of adjacent qubits), sort an order-preserving compression of the
 * key instead.  0 (default) or 1: used where it fits and saves passes; -1:
 * never.  Results are identical either way. */
#define PL_TUNE_WINDOW_KEYS 5
/* L2 prefetch distance of the digit passes, in tiles: each tile's CTA
 * bulk-prefetches into L2 the keys of the tile this many places ahead, so
 * the CTA that later takes that tile reads L2 instead of DRAM.  0 (default):
 * one wave (resident CTAs per SM x SMs); -1: off; k > 0: k tiles.  Results
 * are identical either way. */
#define PL_TUNE_RADIX_PREFETCH 6
/* Look-back window of the digit passes: predecessor tiles read per round
 * trip while a tile waits for its global bucket offsets: 2, 4, 8 or 16; 0
 * (default): 8 for index-packed keys, 4 for key + payload passes.  Results
 * are identical either way. */
#define PL_TUNE_RADIX_WINDOW 7
/* Digit width of a product's index-packed keys: 1: 10-bit digits (1024
 * buckets; a 4096 x 4096 product of 20-qubit strings sorts its 40 varying
 * bits in 4 passes instead of 5) when that saves a pass and the digit pass
 * runs 12 or 16 keys per thread; 0 (default) or -1: 8-bit digits.  Results
 * are identical either way. */
#define PL_TUNE_RADIX_WIDE 8
/* Polls a digit-pass tile makes without progress while it waits for its
 * predecessors' look-back words before each further poll sleeps 64 ns: 1 ..
 * 1024; 0 (default): 16 for index-packed keys, 64 for key + payload passes.  A spinning thread takes issue slots from the
 * warps of other tiles that rank and scatter.  Results are identical either
 * way. */
#define PL_TUNE_RADIX_BACKOFF 9
/* Where canonicalize() of a product takes each sorted term's phase and
 * coefficient: 1: the segment fold gathers them from the operands by the
 * term's index, so the last digit pass moves keys only; 0 (default) or -1:
 * the last digit pass gathers them and writes the coefficients in sorted
 * order.  Results are identical either way. */
#define PL_TUNE_FOLD_GATHER 10
/* Polls a cross-CTA wait (decoupled look-back) makes before it records
 * PL_ERR_TIMEOUT and returns: 1 .. 2^30, 0 = the default 2^20 (with a 64 ns
 * back-off past 64 polls: well under a second).  Written into the device
 * code of the current device; set it again after switching devices. */
#define PL_TUNE_SPIN_LIMIT 3
/* Host-side fault injection: value k > 0 makes the k-th following device
 * allocation of the library fail as if the device were out of memory (the
 * call then reports PL_ERR_OOM); the injection is then spent.  0 = off. */
#define PL_TUNE_FAIL_ALLOC 4
PL_API int pl_set_tuning(int key, int64_t value);
PL_API int pl_get_tuning(int key, int64_t* value);

/* Runs one decoupled look-back wait on a predecessor tile that never
 * publishes (a flag that nothing sets) and stores the status the kernel
 * recorded in *device_status: PL_ERR_TIMEOUT once PL_TUNE_SPIN_LIMIT polls
 * have run out.  Shows on a live device that the library's cross-CTA waits
 * end and leave the context usable.  Synchronous.  No counterpart in the
 * reference (whose kernels do not wait across CTAs). */
PL_API int pl_check_bounded_wait(int* device_status);

/* ---- measurement hooks ------------------------------------------------ */

/* Reset the library's counters.  With enable_timing != 0, every kernel of
 * the collate engine is bracketed by CUDA events recorded on its launching
 * stream (the onesweep digit passes are also summed by pl_profile_read). */
PL_API int pl_profile_reset(int enable_timing);
/* Kernel launches issued by the library since the last reset, and (when
 * timing) the number, total device time and algorithmic bytes (read +
 * write of keys and payloads) of the timed digit passes.  Synchronises the
 * streams the timed passes ran on. */
PL_API int pl_profile_read(uint64_t* launches, uint64_t* timed_launches, double* timed_ms,
                           uint64_t* timed_bytes);
/* Per-kernel totals of every timed launch, one "name count total_ms bytes"
 * line per kernel, into buf (NUL-terminated). */
PL_API int pl_profile_report(char* buf, size_t cap);

#ifdef __cplusplus
}
#endif

#endif /* PAULIB_B200_H */
