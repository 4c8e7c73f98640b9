// Occupied-orbital recovery without an eigensolver.
//
// The reference eigen-decomposes P_eff = X^dagger (S P S * scale) X and keeps the eigenvectors with
// eigenvalue > 0.5 (src/NON_REL/NonRelFockMatrixRi.cpp:96-108, X2C_FockMatrixRi.cpp:109-123,
// UkbFockMatrixRi.cpp:195-209).  The exchange only ever uses the product
//   W = Y_occ diag(w_occ) Y_occ^dagger      (w_occ = 1 for NON_REL, the eigenvalues for X2C/4c),
// so any factor F with F F^dagger = W gives the same K.  Here:
//   1. Pi = step(P_eff - 1/2), the spectral projector onto eigenvalues > 1/2, by the Newton-Schulz
//      sign iteration A <- A (3 - A^2)/2 on A = 2 P_eff - 1 (FP64 DMMA GEMMs only; for an
//      idempotent density A^2 = 1 already and one refinement step is all that runs);
//   2. W = Pi (NON_REL) or Pi P_eff Pi (weighted);
//   3. F = pivoted Cholesky of W (rank r = round(trace Pi) = number of eigenvalues > 1/2), one
//      CTA, left-looking, deterministic;
//   4. c_t = F^dagger X^dagger (r x n), the reference's c_t up to a unitary mixing of the occupied
//      rows, which K is invariant to.
// One host read of r is the only synchronisation.
#include <cfloat>

#include "ri_store.cuh"

namespace rr {

namespace {

// A = 2 Pe - I  (PL = 1 real, 2 interleaved complex).
template <int PL>
__global__ void ns_init_kernel(double* A, const double* Pe, int64_t n) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < n * n;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx / n, j = idx % n;
    A[idx * PL] = 2.0 * Pe[idx * PL] - (i == j ? 1.0 : 0.0);
    if (PL == 2) A[idx * PL + 1] = 2.0 * Pe[idx * PL + 1];
  }
}

__device__ __forceinline__ void atomic_max_pos(double* addr, double v) {
  // v >= 0: IEEE order of non-negative doubles equals the order of their bit patterns.
  atomicMax(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(__double_as_longlong(v)));
}

// out[0] = max |T - I|, out[1] = max_i sum_j |T_ij|  (out zeroed by the caller).
template <int PL>
__global__ void ns_residual_kernel(const double* T, int64_t n, double* out) {
  __shared__ double red0[32], red1[32];
  double m0 = 0.0, m1 = 0.0;
  for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
    double rs = 0.0;
    for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
      const double re = T[(i * n + j) * PL] - (i == j ? 1.0 : 0.0);
      const double im = PL == 2 ? T[(i * n + j) * PL + 1] : 0.0;
      const double a = PL == 2 ? sqrt(re * re + im * im) : fabs(re);
      m0 = fmax(m0, a);
      const double tre = T[(i * n + j) * PL];
      rs += PL == 2 ? sqrt(tre * tre + im * im) : fabs(tre);
    }
    for (int o = 16; o > 0; o >>= 1) rs += __shfl_xor_sync(0xffffffffu, rs, o);
    if ((threadIdx.x & 31) == 0) red1[threadIdx.x >> 5] = rs;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += red1[w];
      m1 = fmax(m1, t);
    }
    __syncthreads();
  }
  for (int o = 16; o > 0; o >>= 1) m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, o));
  if ((threadIdx.x & 31) == 0) red0[threadIdx.x >> 5] = m0;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t = fmax(t, red0[w]);
    atomic_max_pos(out, t);
    atomic_max_pos(out + 1, m1);
  }
}

// Pi = (I + A) / 2, in place on A.
template <int PL>
__global__ void projector_kernel(double* A, int64_t n) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < n * n;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx / n, j = idx % n;
    A[idx * PL] = 0.5 * (A[idx * PL] + (i == j ? 1.0 : 0.0));
    if (PL == 2) A[idx * PL + 1] *= 0.5;
  }
}

constexpr int PC_THREADS = 1024;

// Left-looking pivoted Cholesky of a Hermitian PSD W (n x n, row-major, interleaved when PL = 2):
// W = L L^dagger with L stored TRANSPOSED, Lt (rmax x n, row k = column k of L), so column writes
// and the per-row dot products read coalesced.  The target rank is round(trace(Pi)); the loop also
// stops when the largest remaining diagonal drops below tol * its initial maximum.
// rank_out[0] = rank reached; rows >= rank of Lt are zeroed.  smem: d[n], used[n].
template <int PL>
__global__ void __launch_bounds__(PC_THREADS) pivchol_kernel(const double* W, const double* Pi, int64_t n, double* Lt,
                                                             int64_t rmax, double tol, int* rank_out) {
  extern __shared__ double sm[];
  double* d = sm;
  double* used = sm + n;
  __shared__ double rv[32];
  __shared__ int ri[32];
  __shared__ double s_dmax0, s_dp;
  __shared__ int s_target, s_p;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double tr = 0.0;
  double bv = -DBL_MAX;
  int bi = -1;
  for (int64_t i = tid; i < n; i += PC_THREADS) {
    d[i] = W[(i * n + i) * PL];
    used[i] = 0.0;
    tr += Pi[(i * n + i) * PL];
    if (d[i] > bv) { bv = d[i]; bi = static_cast<int>(i); }
  }
  for (int o = 16; o > 0; o >>= 1) tr += __shfl_xor_sync(0xffffffffu, tr, o);
  if (lane == 0) rv[warp] = tr;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < PC_THREADS / 32; ++w) t += rv[w];
    s_target = max(0, min(static_cast<int>(llrint(t)), static_cast<int>(rmax)));
  }
  __syncthreads();
  const int target = s_target;
  int k = 0;
  for (; k < target; ++k) {
    // block argmax of the thread-local candidates (smallest index on ties)
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov > bv || (ov == bv && oi >= 0 && (bi < 0 || oi < bi))) { bv = ov; bi = oi; }
    }
    if (lane == 0) { rv[warp] = bv; ri[warp] = bi; }
    __syncthreads();
    if (tid == 0) {
      double v = -DBL_MAX;
      int ix = -1;
      for (int w = 0; w < PC_THREADS / 32; ++w)
        if (rv[w] > v || (rv[w] == v && ri[w] >= 0 && (ix < 0 || ri[w] < ix))) { v = rv[w]; ix = ri[w]; }
      if (k == 0) s_dmax0 = v;
      s_p = ix;
      s_dp = v;
      if (ix >= 0) used[ix] = 1.0;
    }
    __syncthreads();
    const int p = s_p;
    const double dp = s_dp;
    if (p < 0 || !(dp > tol * s_dmax0) || !(dp > 0.0)) break;
    const double inv = rsqrt(dp);
    bv = -DBL_MAX;
    bi = -1;
    for (int64_t i = tid; i < n; i += PC_THREADS) {
      // column p of W = conj(row p) for a Hermitian W (row p is contiguous)
      double cr = W[(p * n + i) * PL];
      double ci = PL == 2 ? -W[(p * n + i) * PL + 1] : 0.0;
      for (int j = 0; j < k; ++j) {
        const double* lj = Lt + j * n * PL;
        if (PL == 2) {  // c -= L[i][j] * conj(L[p][j])
          const double ar = lj[2 * i], ai = lj[2 * i + 1], br = lj[2 * p], bi2 = lj[2 * p + 1];
          cr -= ar * br + ai * bi2;
          ci -= ai * br - ar * bi2;
        } else {
          cr -= lj[i] * lj[p];
        }
      }
      double* out = Lt + (k * n + i) * PL;
      out[0] = cr * inv;
      if (PL == 2) out[1] = ci * inv;
      const double di = d[i] - (cr * cr + ci * ci) / dp;
      d[i] = di;
      if (used[i] == 0.0 && di > bv) { bv = di; bi = static_cast<int>(i); }
    }
    // Lt row k is read by every thread in the next step: make the writes visible block-wide.
    __syncthreads();
  }
  for (int64_t idx = tid; idx < (rmax - k) * n * PL; idx += PC_THREADS) Lt[k * n * PL + idx] = 0.0;
  if (tid == 0) rank_out[0] = k;
}

int blocks_for(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 1184))); }

}  // namespace

// Recovers c_t (r x n, row-major) from the density.  cplx selects interleaved complex matrices;
// weighted multiplies the projector by P_eff (sqrt(occupation) weighting of X2C / 4c).
// Dp: density (n x n, ld n); S (n x n); X (n x n_eff).  Returns r.
int64_t occupied_ct(rr_ri_store* h, const double* X, const double* S, const double* Dp, int64_t n, int64_t n_eff,
                    double scale, bool cplx, bool weighted, double* Ct, cudaStream_t s) {
  const int PL = cplx ? 2 : 1;
  if (n_eff == 0) return 0;
  double *SD, *SDS, *Y, *Pe, *A, *T, *A2, *F, *res;
  int* rank;
  Arena ar(&h->solver_a);
  ar.request(&SD, n * n * PL);
  ar.request(&SDS, n * n * PL);
  ar.request(&Y, n * n_eff * PL);
  ar.request(&Pe, n_eff * n_eff * PL);
  ar.request(&A, n_eff * n_eff * PL);
  ar.request(&T, n_eff * n_eff * PL);
  ar.request(&A2, n_eff * n_eff * PL);
  ar.request(&F, n_eff * n_eff * PL);
  ar.request(&res, 4);
  ar.commit();
  rank = reinterpret_cast<int*>(res + 2);

  // Small GEMMs split K across the GPU: give them the handle's scratch.
  h->work.ensure(static_cast<size_t>(std::max<int64_t>(static_cast<int64_t>(h->work.n), 8 * n * n * PL)));
  double* wk = h->work.p;
  const int64_t wcap = static_cast<int64_t>(h->work.n);
  // P_eff = X^dagger (S D S * scale) X
  GemmDesc g;
  g.cplx = cplx;
  g.M = n; g.N = n; g.K = n;
  g.A = S; g.lda = n; g.B = Dp; g.ldb = n; g.C = SD; g.ldc = n;
  gemm(g, s, wk, wcap);
  g.A = SD; g.B = S; g.C = SDS;
  gemm(g, s, wk, wcap);
  g.N = n_eff; g.A = SDS; g.B = X; g.ldb = n_eff; g.C = Y; g.ldc = n_eff;
  gemm(g, s, wk, wcap);
  GemmDesc pe;
  pe.cplx = cplx;
  pe.M = n_eff; pe.N = n_eff; pe.K = n;
  pe.A = X; pe.lda = n_eff; pe.opA = Op::T; pe.conjA = cplx;
  pe.B = Y; pe.ldb = n_eff; pe.C = Pe; pe.ldc = n_eff; pe.alpha = scale;
  gemm(pe, s, wk, wcap);

  // Newton-Schulz sign iteration on A = 2 Pe - I.
  if (cplx) ns_init_kernel<2><<<blocks_for(n_eff * n_eff), 256, 0, s>>>(A, Pe, n_eff);
  else ns_init_kernel<1><<<blocks_for(n_eff * n_eff), 256, 0, s>>>(A, Pe, n_eff);
  RR_LAUNCH_CHECK();
  GemmDesc sq;
  sq.cplx = cplx;
  sq.M = n_eff; sq.N = n_eff; sq.K = n_eff;
  sq.lda = n_eff; sq.ldb = n_eff; sq.ldc = n_eff;
  double hres[2] = {0.0, 0.0};
  bool converged = false;
  const int max_iter = 100;
  for (int it = 0; it < max_iter; ++it) {
    sq.A = A; sq.B = A; sq.C = T; sq.alpha = 1.0;
    gemm(sq, s, wk, wcap);
    RR_CUDA(cudaMemsetAsync(res, 0, 2 * sizeof(double), s));
    if (cplx) ns_residual_kernel<2><<<static_cast<int>(std::min<int64_t>(n_eff, 592)), 256, 0, s>>>(T, n_eff, res);
    else ns_residual_kernel<1><<<static_cast<int>(std::min<int64_t>(n_eff, 592)), 256, 0, s>>>(T, n_eff, res);
    RR_LAUNCH_CHECK();
    RR_CUDA(cudaMemcpyAsync(hres, res, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    RR_CUDA(cudaStreamSynchronize(s));
    if (it == 0 && hres[1] > 2.5) {
      // ||A||_2 <= sqrt(||A^2||_inf): scale into the convergence region of the iteration
      axpby(A, A, 0.0, 1.0 / std::sqrt(hres[1]), n_eff * n_eff * PL, s);
      continue;
    }
    // A <- 1.5 A - 0.5 A T (always at least one refinement step)
    sq.A = A; sq.B = T; sq.C = A2; sq.alpha = 1.0;
    gemm(sq, s, wk, wcap);
    axpby(A, A2, -0.5, 1.5, n_eff * n_eff * PL, s);
    if (hres[0] < 1e-10) { converged = true; break; }
  }
  RR_REQUIRE(converged, RR_ERR_SOLVER,
             "occupied recovery: an eigenvalue of X^dagger(SPS)X sits at the 0.5 threshold (sign iteration did not converge)");
  if (cplx) projector_kernel<2><<<blocks_for(n_eff * n_eff), 256, 0, s>>>(A, n_eff);
  else projector_kernel<1><<<blocks_for(n_eff * n_eff), 256, 0, s>>>(A, n_eff);
  RR_LAUNCH_CHECK();
  const double* W = A;
  if (weighted) {  // W = Pi Pe Pi
    sq.A = A; sq.B = Pe; sq.C = T;
    gemm(sq, s, wk, wcap);
    sq.A = T; sq.B = A; sq.C = A2;
    gemm(sq, s, wk, wcap);
    W = A2;
  }
  const size_t smem = sizeof(double) * 2 * n_eff;
  RR_REQUIRE(smem <= 200 * 1024, RR_ERR_ARG, "occupied recovery: n_eff too large for the pivoted Cholesky kernel");
  if (cplx) {
    auto k = pivchol_kernel<2>;
    RR_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    k<<<1, PC_THREADS, smem, s>>>(W, A, n_eff, F, n_eff, 1e-12, rank);
  } else {
    auto k = pivchol_kernel<1>;
    RR_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    k<<<1, PC_THREADS, smem, s>>>(W, A, n_eff, F, n_eff, 1e-12, rank);
  }
  RR_LAUNCH_CHECK();
  int r = 0;
  RR_CUDA(cudaMemcpyAsync(&r, rank, sizeof(int), cudaMemcpyDeviceToHost, s));
  RR_CUDA(cudaStreamSynchronize(s));
  if (r == 0) return 0;
  // c_t = F^dagger X^dagger = conj(Lt) X^dagger  (r x n)
  GemmDesc ct;
  ct.cplx = cplx;
  ct.M = r; ct.N = n; ct.K = n_eff;
  ct.A = F; ct.lda = n_eff; ct.opA = Op::N; ct.conjA = cplx;
  ct.B = X; ct.ldb = n_eff; ct.opB = Op::T; ct.conjB = cplx;
  ct.C = Ct; ct.ldc = n;
  gemm(ct, s, wk, wcap);
  return r;
}

}  // namespace rr
