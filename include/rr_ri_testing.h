/* librr_ri test hooks: direct access to the internal kernel families for unit tests.
 * All pointers are DEVICE pointers; calls are synchronous.  No reference counterpart: these
 * exist so the DMMA GEMM and the J streaming passes can be checked in isolation. */
#ifndef RR_RI_TESTING_H
#define RR_RI_TESTING_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* C[b] = alpha op(A[b]) op(B[b]) + beta C[b] on the FP64 DMMA GEMM (row-major; op 0 = N, 1 = T;
 * cplx: interleaved complex; mirror +1/-1 fills the strict lower triangle from the upper one;
 * allow_split lets the kernel split K with a deterministic reduction). */
int rr_test_gemm_f64(int64_t M, int64_t N, int64_t K, const double* A, int64_t lda, int64_t strideA, int32_t opA,
                     const double* B, int64_t ldb, int64_t strideB, int32_t opB, double* C, int64_t ldc,
                     int64_t strideC, double alpha, double beta, int64_t batch, int32_t cplx, int32_t conjA,
                     int32_t conjB, int32_t mirror, int32_t allow_split);

/* gamma = B vec(D) and J = B^T gamma through the TMA streaming passes (B: naux x n2, dense). */
int rr_test_j_passes(const double* B, int64_t naux, int64_t n2, const double* D, double* gamma, double* J);

/* The same passes over the packed upper triangles of the n x n rows of B (the store's J path when
 * every B^P is symmetric to a few ulps): *packed = 1 when B passed the symmetry test and the packed
 * passes ran, 0 when the dense passes ran instead (D, J: n x n). */
int rr_test_j_passes_packed(const double* B, int64_t naux, int64_t n, const double* D, double* gamma, double* J,
                            int32_t* packed);

/* K = sum_P (Ct B^P)^T (Ct B^P) through the split-BF16 tcgen05 exchange (B: naux x n*n dense,
 * Ct: nocc x n, K: n x n; all FP64 device pointers). */
int rr_test_mixed_exchange(const double* B, int64_t naux, int64_t n, const double* Ct, int64_t nocc, double* K);

/* dK = K(Ct) - K(Ct_prev) through the incremental split-BF16 exchange:
 * sum_P (W B^P)^T (U B^P) + (U B^P)^T (W B^P), W = (Ct + Ct_prev)/2, U = Ct - Ct_prev (device pointers). */
int rr_test_mixed_exchange_delta(const double* B, int64_t naux, int64_t n, const double* Ct, const double* Ct_prev,
                                 int64_t nocc, double* dK);

/* Adam<T>::step (src/Utils/ADAM.cpp:33-51) on the device over `nsteps` host gradients (rows of
 * grads, n entries, interleaved complex when cplx); steps receives the nsteps x n updates. */
int rr_test_adam_steps(int64_t n, int32_t cplx, int64_t nsteps, double lr, double b1, double b2, double eps,
                       const double* grads, double* steps);

/* exp(-kappa) of a real antisymmetric n x n host matrix by the device scaling-and-squaring route the
 * orbital optimiser uses (src/Hessian_opt/SpinorRotation.cpp:17 computes the same matrix). */
int rr_test_rotation_matrix(int64_t n, const double* kappa, double* U);

/* The same for an anti-Hermitian complex kappa (interleaved n x n host matrices in and out), the
 * route of the complex orbital optimiser. */
int rr_test_rotation_matrix_complex(int64_t n, const double* kappa, double* U);

/* AdamOptimizer<double>::run `runs` times (ADAM.cpp:140-213) on E(x) = sum (a x^2 / 2 + b x) +
 * c (sum x^2)^2 with x += step, driven by the device ADAM and the library's run logic. */
int rr_test_adam_run_quadratic(int64_t n, const double* a, const double* b, double c, const double* x0, int32_t runs,
                               double* energy_best, int32_t* iterations, int32_t* restart, double* rate,
                               double* x_out);

/* Number of device allocations (cudaMalloc of the library's own buffers) made by this process so far:
 * a call that allocates nothing leaves it unchanged. */
int64_t rr_test_device_allocations(void);

/* T[P] = Ct B^P for P < naux (Ct nocc x n, B naux x n^2, T naux x nocc x n; device pointers, synchronous)
 * through the general DMMA GEMM (variant 0, m8n8k4) or the m16n8k8 half-transform (variant 1: its default
 * tiling; 2-14: the alternative tilings kept for measurement). */
int rr_test_half_transform(const double* Ct, int64_t nocc, const double* B, int64_t naux, int64_t n, double* T,
                           int32_t variant);
/* The same, `reps` times after one warm-up; *ms = the average device time of one (CUDA events). */
int rr_test_half_transform_time(const double* Ct, int64_t nocc, const double* B, int64_t naux, int64_t n, double* T,
                                int32_t variant, int32_t reps, double* ms);

/* Failure detection without a fault: one CTA of `threads` threads waits on an mbarrier that nothing
 * arrives on (and no bulk copy is in flight) through the bounded wait every TMA pipeline of the library
 * uses, with `spin_limit` polls (1 .. 4,194,304, the pipelines' own limit).  The wait expires, records
 * its code in the status word and returns; the hook then returns RR_ERR_TIMEOUT, as a pipeline call
 * does.  status_word: the recorded code; elapsed_ms: the launch's device time (CUDA events);
 * cycles: SM clock cycles thread 0 spent in the wait. */
int rr_test_wait_expiry(uint32_t spin_limit, int32_t threads, int32_t* status_word, double* elapsed_ms,
                        double* cycles);

/* The device Boys function of the integral kernels: out[i (nmax+1) + n] = F_n(T[i]) for n <= nmax <= 18
 * (host arrays). */
int rr_test_boys(const double* T, int64_t count, int32_t nmax, double* out);

#ifdef __cplusplus
}
#endif

#endif /* RR_RI_TESTING_H */
