// Occupied-orbital recovery without an eigensolver.
//
// The reference eigen-decomposes P_eff = X^dagger (S P S * scale) X and keeps the eigenvectors with
// eigenvalue > 0.5 (src/NON_REL/NonRelFockMatrixRi.cpp:96-108, X2C_FockMatrixRi.cpp:109-123,
// UkbFockMatrixRi.cpp:195-209).  The exchange only ever uses the product
//   W = Y_occ diag(w_occ) Y_occ^dagger      (w_occ = 1 for NON_REL, the eigenvalues for X2C/4c),
// so any factor F with F F^dagger = W gives the same K.  Here:
//   1. Pi = step(P_eff - 1/2), the spectral projector onto eigenvalues > 1/2, by the Newton-Schulz
//      sign iteration A <- A (3 - A^2)/2 on A = 2 P_eff - 1 (FP64 DMMA GEMMs only; for an
//      idempotent density A^2 = 1 already to rounding and the iteration stops at its first check);
//   2. W = Pi (NON_REL) or Pi P_eff Pi (weighted);
//   3. an orthonormal basis Q of range(Pi) (rank r = trace Pi = number of eigenvalues > 1/2) by
//      CholeskyQR2 of Pi G for a fixed pseudo-random G (deterministic), and F = Q for NON_REL or
//      F = Q chol(Q^dagger P_eff Q) for the weighted case, so F F^dagger = W;
//   4. c_t = F^dagger X^dagger (r x n), the reference's c_t up to a unitary mixing of the occupied
//      rows, which K is invariant to.
// The Newton-Schulz residual read-back (which also yields trace Pi) is the only synchronisation.
#include <cfloat>

#include "chol.cuh"
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

// out[0] = max |T - I|, out[1] = max_i sum_j |T_ij|, out[2] += Re trace(A)  (out zeroed by the caller).
template <int PL>
__global__ void ns_residual_kernel(const double* T, const double* A, int64_t n, double* out) {
  __shared__ double red0[32], red1[32];
  double m0 = 0.0, m1 = 0.0;
  if (threadIdx.x == 0) {
    double tr = 0.0;
    for (int64_t i = blockIdx.x; i < n; i += gridDim.x) tr += A[(i * n + i) * PL];
    atomicAdd(out + 2, tr);
  }
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

// Deterministic pseudo-random test matrix G (rows x cols, interleaved when PL = 2), entries in
// [-1, 1) from a 64-bit integer hash of the index (splitmix64).
template <int PL>
__global__ void fill_test_matrix_kernel(double* G, int64_t count) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < count * PL;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint64_t z = static_cast<uint64_t>(idx) + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    G[idx] = static_cast<double>(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
  }
}

// SMEM selects the buffer at compile time, so the shared-memory variant addresses it with
// shared-memory instructions (a pointer that may be either compiles to slower generic accesses).
template <int PL, bool SMEM>
__global__ void __launch_bounds__(CHOL_THREADS) chol_block_kernel(const double* M, int r, double* out,
                                                                  int want_inverse, int* status, double* gbuf) {
  extern __shared__ double sm[];
  chol_block_body<PL>(M, r, out, want_inverse, status, SMEM ? sm : gbuf);
}

int blocks_for(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 1184))); }

}  // namespace

// From a rank-r orthogonal projector Pi (n_eff x n_eff, in the orthonormal basis of X) build
// c_t = F^dagger X^dagger (r x n, leading dim n) with F F^dagger = Pi (Pe == nullptr) or
// Pi Pe Pi (weighted): Y = Pi G for a fixed pseudo-random G, CholeskyQR2, optional weighting.
void projector_ct(rr_ri_store* h, const double* A, const double* Pe, const double* X, int64_t n, int64_t n_eff,
                  int64_t r, bool cplx, double* Ct, cudaStream_t s) {
  const int PL = cplx ? 2 : 1;
  const bool weighted = Pe != nullptr;
  if (r == 0) return;
  h->work.ensure(static_cast<size_t>(std::max<int64_t>(static_cast<int64_t>(h->work.n), 8 * n * n * PL)));
  double* wk = h->work.p;
  const int64_t wcap = static_cast<int64_t>(h->work.n);
  // Orthonormal basis of range(Pi): Y = Pi G (fixed pseudo-random G), CholeskyQR2 with the small
  // triangular factors applied as GEMMs.
  double *G, *Y2, *Y3, *M, *Wt, *PQ, *gw;
  Arena ar2(&h->T);  // the exchange intermediate is not live yet
  ar2.request(&G, n_eff * r * PL);
  ar2.request(&Y2, n_eff * r * PL);
  ar2.request(&Y3, n_eff * r * PL);
  ar2.request(&M, r * r * PL);
  ar2.request(&Wt, r * r * PL);
  ar2.request(&PQ, n_eff * r * PL);
  ar2.request(&gw, 2 * r * (r | 1) * PL + r);
  ar2.commit();
  // factor + inverse + pivots in shared memory when they fit, else in the global scratch gw
  const size_t block_smem = sizeof(double) * (2 * r * (r | 1) * PL + r);
  const bool chol_in_smem = block_smem <= 227 * 1024;
  if (cplx) fill_test_matrix_kernel<2><<<blocks_for(n_eff * r * 2), 256, 0, s>>>(G, n_eff * r);
  else fill_test_matrix_kernel<1><<<blocks_for(n_eff * r), 256, 0, s>>>(G, n_eff * r);
  RR_LAUNCH_CHECK();
  GemmDesc y;
  y.cplx = cplx;
  y.M = n_eff; y.N = r; y.K = n_eff;
  y.A = A; y.lda = n_eff; y.B = G; y.ldb = r; y.C = Y2; y.ldc = r;
  gemm(y, s, wk, wcap);
  auto chol = [&](const double* mat, int inverse) {
    const int sm = chol_in_smem ? static_cast<int>(block_smem) : 0;
    auto k = cplx ? (chol_in_smem ? chol_block_kernel<2, true> : chol_block_kernel<2, false>)
                  : (chol_in_smem ? chol_block_kernel<1, true> : chol_block_kernel<1, false>);
    if (sm > 48 * 1024) RR_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    k<<<1, CHOL_THREADS, sm, s>>>(mat, static_cast<int>(r), Wt, inverse, h->status.p + 1, chol_in_smem ? nullptr : gw);
    RR_LAUNCH_CHECK();
  };
  GemmDesc gm;  // M = Y^dagger Y
  gm.cplx = cplx;
  gm.M = r; gm.N = r; gm.K = n_eff;
  gm.opA = Op::T; gm.conjA = cplx; gm.lda = r; gm.ldb = r; gm.C = M; gm.ldc = r;
  GemmDesc yw;  // Y_out = Y_in Wt
  yw.cplx = cplx;
  yw.M = n_eff; yw.N = r; yw.K = r;
  yw.lda = r; yw.B = Wt; yw.ldb = r; yw.ldc = r;
  double* cur = Y2;
  double* nxt = Y3;
  for (int pass = 0; pass < 2; ++pass) {
    gm.A = cur; gm.B = cur;
    gemm(gm, s, wk, wcap);
    chol(M, 1);
    yw.A = cur; yw.C = nxt;
    gemm(yw, s, wk, wcap);
    std::swap(cur, nxt);
  }
  if (weighted) {  // F = Q chol(Q^dagger Pe Q): F F^dagger = Pi Pe Pi
    GemmDesc pq;
    pq.cplx = cplx;
    pq.M = n_eff; pq.N = r; pq.K = n_eff;
    pq.A = Pe; pq.lda = n_eff; pq.B = cur; pq.ldb = r; pq.C = PQ; pq.ldc = r;
    gemm(pq, s, wk, wcap);
    gm.A = cur; gm.B = PQ;
    gemm(gm, s, wk, wcap);
    chol(M, 0);
    yw.A = cur; yw.C = nxt;
    gemm(yw, s, wk, wcap);
    std::swap(cur, nxt);
  }
  Y2 = cur;
  // c_t = F^dagger X^dagger  (r x n)
  GemmDesc ct;
  ct.cplx = cplx;
  ct.M = r; ct.N = n; ct.K = n_eff;
  ct.A = Y2; ct.lda = r; ct.opA = Op::T; ct.conjA = cplx;
  ct.B = X; ct.ldb = n_eff; ct.opB = Op::T; ct.conjB = cplx;
  ct.C = Ct; ct.ldc = n;
  gemm(ct, s, wk, wcap);
}

// Recovers c_t (r x n, row-major) from the density.  cplx selects interleaved complex matrices;
// weighted multiplies the projector by P_eff (sqrt(occupation) weighting of X2C / 4c).
// Dp: density (n x n, ld n); S (n x n); X (n x n_eff).  d_ready (optional): event s waits on
// before the first product that reads Dp.  Returns r.
int64_t occupied_ct(rr_ri_store* h, const double* X, const double* S, const double* Dp, int64_t n, int64_t n_eff,
                    double scale, bool cplx, bool weighted, double* Ct, cudaStream_t s, cudaEvent_t d_ready) {
  const int PL = cplx ? 2 : 1;
  if (n_eff == 0) return 0;
  double *SD, *Y, *Pe, *A, *T, *A2, *F, *res;
  int* rank;
  Arena ar(&h->solver_a);
  ar.request(&SD, n * n_eff * PL);
  ar.request(&Y, n * n_eff * PL);
  ar.request(&Pe, n_eff * n_eff * PL);
  ar.request(&A, n_eff * n_eff * PL);
  ar.request(&T, n_eff * n_eff * PL);
  ar.request(&A2, n_eff * n_eff * PL);
  ar.request(&F, n_eff * n_eff * PL);
  ar.request(&res, 8);
  ar.commit();
  rank = reinterpret_cast<int*>(res + 4);
  (void)rank;

  // Small GEMMs split K across the GPU: give them the handle's scratch.
  h->work.ensure(static_cast<size_t>(std::max<int64_t>(static_cast<int64_t>(h->work.n), 8 * n * n * PL)));
  double* wk = h->work.p;
  const int64_t wcap = static_cast<int64_t>(h->work.n);
  // P_eff = X^dagger (S D S * scale) X = Z^dagger D Z * scale with Z = S X (S is Hermitian): three
  // products instead of four.
  GemmDesc g;
  g.cplx = cplx;
  g.M = n; g.N = n_eff; g.K = n;
  g.A = S; g.lda = n; g.B = X; g.ldb = n_eff; g.C = SD; g.ldc = n_eff;  // Z (n x n_eff) in SD
  gemm(g, s, wk, wcap);
  if (d_ready) RR_CUDA(cudaStreamWaitEvent(s, d_ready, 0));  // D may still be arriving from the host
  g.A = Dp; g.B = SD; g.C = Y;  // Y = D Z
  gemm(g, s, wk, wcap);
  GemmDesc pe;
  pe.cplx = cplx;
  pe.M = n_eff; pe.N = n_eff; pe.K = n;
  pe.A = SD; pe.lda = n_eff; pe.opA = Op::T; pe.conjA = cplx;
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
  double hres[3] = {0.0, 0.0, 0.0};
  bool converged = false;
  const int max_iter = 100;
  for (int it = 0; it < max_iter; ++it) {
    sq.A = A; sq.B = A; sq.C = T; sq.alpha = 1.0;
    gemm(sq, s, wk, wcap);
    RR_CUDA(cudaMemsetAsync(res, 0, 3 * sizeof(double), s));
    if (cplx) ns_residual_kernel<2><<<static_cast<int>(std::min<int64_t>(n_eff, 592)), 256, 0, s>>>(T, A, n_eff, res);
    else ns_residual_kernel<1><<<static_cast<int>(std::min<int64_t>(n_eff, 592)), 256, 0, s>>>(T, A, n_eff, res);
    RR_LAUNCH_CHECK();
    RR_CUDA(cudaMemcpyAsync(hres, res, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    host_wait(h, s);
    if (it == 0 && hres[1] > 2.5) {
      // ||A||_2 <= sqrt(||A^2||_inf): scale into the convergence region of the iteration
      axpby(A, A, 0.0, 1.0 / std::sqrt(hres[1]), n_eff * n_eff * PL, s);
      continue;
    }
    // A density that is a projector to rounding (an SCF density) gives A^2 = I already: A is the
    // sign, and a refinement would only move it by rounding.  Otherwise A <- 1.5 A - 0.5 A T.
    if (hres[0] < 1e-13) { converged = true; break; }
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
  // Rank = number of eigenvalues above 1/2 = trace(Pi) = (n_eff + trace(sign))/2.
  const int64_t r = std::max<int64_t>(0, std::min<int64_t>(n_eff, std::llround(0.5 * (n_eff + hres[2]))));
  if (r == 0) return 0;
  projector_ct(h, A, weighted ? Pe : nullptr, X, n, n_eff, r, cplx, Ct, s);
  return r;
}

}  // namespace rr
