// Small dense Cholesky factorisation (with optional inverse) in one CTA: the CholeskyQR steps of the
// occupied-orbital recovery and of the grouped SCF loops.
#pragma once

#include "rr_common.cuh"

namespace rr {

// Cholesky M = L L^dagger of a small Hermitian positive-definite r x r matrix (row-major,
// interleaved when PL = 2).  Output: out = L^{-dagger} (want_inverse) or L (upper triangle zero),
// r x r row-major, so that Y <- Y out is a plain GEMM.  status[0] |= 1 on a non-positive pivot.
// One CTA of CHOL_THREADS threads; the factor, the inverse and the pivots live in shared memory, or
// in `gbuf` (global, 2 r (r|1) PL + r doubles, L2-resident at these sizes) when they do not fit.  One
// __syncthreads per elimination step:
//  * step j of the factorisation updates the trailing triangle with the UNSCALED column j
//    (A[i][k] -= A[i][j] conj(A[k][j]) / d_j, spread over all threads) and, in the same phase,
//    finishes column j-1 (scale by 1/sqrt(d), set the diagonal), which nothing reads any more;
//  * the inverse is forward elimination on X = I with the same one-phase-per-row scheme.
constexpr int CHOL_THREADS = 256;  // 16 x 16: the element updates use a 2-D thread grid

// The body, run by all CHOL_THREADS threads of the calling CTA; buf: the CTA's dynamic shared memory
// or the global scratch.  Inlined into its kernels, so the shared-memory variant addresses the buffer
// with shared-memory instructions.
template <int PL>
__device__ __forceinline__ void chol_block_body(const double* M, int r, double* out, int want_inverse, int* status,
                                                double* buf) {
  // Row pitch ld = r | 1 elements: a column (rows k, k+1, ...) then spreads over all banks instead
  // of hitting one bank per access as with an even pitch (r = 80 complex: 160 doubles per row).
  const int ld = r | 1;
  double* A = buf;                 // r x r (pitch ld), factor in the lower triangle
  double* X = A + r * ld * PL;     // r x r (pitch ld), L^{-1}
  double* piv = X + r * ld * PL;   // r pivots d_j before the square root
  const int t = threadIdx.x, ty = t >> 4, tx = t & 15;  // 16 x 16 grid for the element updates
  for (int i = ty; i < r; i += 16)
    for (int k = tx; k < r; k += 16) {
      A[(i * ld + k) * PL] = M[(i * r + k) * PL];
      if (PL == 2) A[(i * ld + k) * PL + 1] = M[(i * r + k) * PL + 1];
      if (want_inverse) {
        X[(i * ld + k) * PL] = i == k ? 1.0 : 0.0;
        if (PL == 2) X[(i * ld + k) * PL + 1] = 0.0;
      }
    }
  __syncthreads();
  // Phase j runs factorisation step j and, when the inverse is wanted, inverse step j - 2, whose
  // column of L was finished in phase j - 1: r + 3 barriers instead of 2 r + 2.  The two steps touch
  // disjoint data (the factorisation writes columns j - 1 and > j of A, the inverse step reads
  // columns j - 2 and j - 3 of A and writes X).
  const int last = want_inverse ? r + 2 : r;
  for (int j = 0; j <= last; ++j) {
    if (j > 0 && j <= r) {  // finish column j-1 (its pivot was saved in step j-1; nothing reads the column now)
      const int c = j - 1;
      double d = piv[c];
      if (!(d > 0.0)) d = 1e-300;
      const double inv = 1.0 / sqrt(d);
      for (int i = c + 1 + t; i < r; i += CHOL_THREADS) {
        A[(i * ld + c) * PL] *= inv;
        if (PL == 2) A[(i * ld + c) * PL + 1] *= inv;
      }
      if (t == 0) {
        if (!(piv[c] > 0.0)) atomicOr(status, 1);
        A[(c * ld + c) * PL] = sqrt(d);
        if (PL == 2) A[(c * ld + c) * PL + 1] = 0.0;
      }
    }
    if (j < r) {
      double d = A[(j * ld + j) * PL];  // final: step j writes only columns k > j
      if (t == 0) piv[j] = d;
      if (!(d > 0.0)) d = 1e-300;
      const double inv_d = 1.0 / d;
      // trailing triangle rows j+1..r-1, element (i, k) with k <= i: a 16 x 16 thread grid strides
      // over rows (ty) and columns (tx), no index division
      for (int i = j + 1 + ty; i < r; i += 16) {
        const double ar = A[(i * ld + j) * PL] * inv_d, ai = PL == 2 ? A[(i * ld + j) * PL + 1] * inv_d : 0.0;
        for (int k = j + 1 + tx; k <= i; k += 16) {
          const double br = A[(k * ld + j) * PL], bi = PL == 2 ? A[(k * ld + j) * PL + 1] : 0.0;
          A[(i * ld + k) * PL] -= ar * br + ai * bi;
          if (PL == 2) A[(i * ld + k) * PL + 1] -= ai * br - ar * bi;
        }
      }
    }
    // Inverse step q = j - 2 (forward elimination on X = I): row q of X is final once divided by
    // L[q][q]; rows i > q subtract L[i][q] / L[q][q] times the undivided row q (columns c <= q), and
    // row q-1 is divided in the same step.
    const int q = j - 2;
    if (want_inverse && q >= 0) {
      if (q > 0) {
        const int p1 = q - 1;
        const double inv = 1.0 / A[(p1 * ld + p1) * PL];
        for (int c = t; c <= p1; c += CHOL_THREADS) {
          X[(p1 * ld + c) * PL] *= inv;
          if (PL == 2) X[(p1 * ld + c) * PL + 1] *= inv;
        }
      }
      if (q < r) {
        const double inv = 1.0 / A[(q * ld + q) * PL];
        for (int i = q + 1 + ty; i < r; i += 16) {
          const double lr = A[(i * ld + q) * PL] * inv, li = PL == 2 ? A[(i * ld + q) * PL + 1] * inv : 0.0;
          for (int c = tx; c <= q; c += 16) {
            const double xr = X[(q * ld + c) * PL], xi = PL == 2 ? X[(q * ld + c) * PL + 1] : 0.0;
            X[(i * ld + c) * PL] -= lr * xr - li * xi;
            if (PL == 2) X[(i * ld + c) * PL + 1] -= lr * xi + li * xr;
          }
        }
      }
    }
    __syncthreads();
  }
  if (!want_inverse) {
    for (int e = t; e < r * r; e += CHOL_THREADS) {
      const int i = e / r, k = e % r;
      out[e * PL] = k <= i ? A[(i * ld + k) * PL] : 0.0;
      if (PL == 2) out[e * PL + 1] = k <= i ? A[(i * ld + k) * PL + 1] : 0.0;
    }
    return;
  }
  // out = (L^{-1})^dagger: out[c][i] = conj(X[i][c])
  for (int e = t; e < r * r; e += CHOL_THREADS) {
    const int c = e / r, i = e % r;
    out[e * PL] = i >= c ? X[(i * ld + c) * PL] : 0.0;
    if (PL == 2) out[e * PL + 1] = i >= c ? -X[(i * ld + c) * PL + 1] : 0.0;
  }
}

}  // namespace rr
