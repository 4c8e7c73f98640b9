// Device-resident RHF SCF loop over the RI Fock build (reference: nonRelScfImpl,
// src/NON_REL/NonRelHartreeFock.cpp:117-198, and Diis<T>, src/Utils/DIIS.cpp:53-131).
//
// Per iteration, everything but a 6x6 DIIS solve stays on the GPU:
//   F = h + J(P) - K(C_occ)         (J FP64; K FP64 DMMA or split-BF16 tcgen05 by phase)
//   E = 1/2 Tr[P (h + F)]           (the un-extrapolated F, as the reference)
//   e = F P S - S P F, DIIS extrapolation (newest-first history, scaled B, bordered solve,
//   drop-oldest on a singular system: the reference's algorithm, solved on the host)
//   F_ortho = X^T F_scf X, then the aufbau projector onto its lowest nocc eigenvectors by SP2
//   trace-correcting purification (GEMMs only; no eigensolver), C_occ from the projector
//   P_new = 2 C_occ C_occ^T; converged when dP < tolP OR dE < tolE (from the second iteration).
// The first iteration builds F from the caller's start density through the drop-in Fock build
// (occupied recovery included); later iterations reuse the loop's own C_occ.
//
// Mixed precision (RR_PREC_MIXED): an incremental split-BF16 exchange (the exchange of the change
// of the occupied orbitals is added to the previous one, so the rounding error follows the density
// change), J in FP64, and one FP64 build of the converged density for the reported energy.
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "ri_store.cuh"

namespace rr {

void exchange_nonrel(rr_ri_store* h, const double* Ct, int64_t ldct, bool ct_transposed, int64_t nocc, double* K,
                     cudaStream_t s, const double* Dp, double* Jout, bool half_only = false);
void energy_nonrel(rr_ri_store* h, const double* Ct, int64_t nocc, const double* Dp, double* Jout, double* energy,
                   cudaStream_t s);
void coulomb_after_ht(rr_ri_store* h, const double* Dp, const double* Ct, int64_t nocc, double* J, const double* tgam,
                      int tseg, cudaStream_t s);
void coulomb_join(rr_ri_store* h, cudaStream_t s);
void fock_nonrel(rr_ri_store* h, const double* hc, const double* D, const double* S, const double* X, int64_t n_eff,
                 double* F, const rr_opts* o);
void projector_ct(rr_ri_store* h, const double* A, const double* Pe, const double* X, int64_t n, int64_t n_eff,
                  int64_t r, bool cplx, double* Ct, cudaStream_t s);
void fock_x2c(rr_ri_store* h, const double* hc, const double* P, const double* S, const double* X, int64_t n_eff,
              double* F, const rr_opts* o, const RelBuild* rb = nullptr, const double* proj = nullptr,
              int64_t proj_rank = 0);
void fock_rkb(rr_ri_store* h, const double* hc, const double* v, int64_t n_rkb, const double* s_full,
              const double* x_full, int64_t n_eff, const double* P, double* F, const rr_opts* o,
              const RelBuild* rb = nullptr, const double* proj = nullptr, int64_t proj_rank = 0);

namespace {

int blocks_for(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 1184))); }

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += red[w];
  __syncthreads();
  return t;
}

// Two-stage reductions: RED_CTAS CTAs write one partial each (CTA b owns a fixed chunk), then one
// CTA per row combines the partials in a fixed order, so sums are identical run to run.
constexpr int RED_CTAS = 256;

template <int OP>  // 0 sum, 1 min, 2 max
__global__ void reduce_partials_kernel(const double* part, int cols, double scale, double* out) {
  __shared__ double red[32];
  const double* row = part + static_cast<int64_t>(blockIdx.x) * cols;
  double v = OP == 0 ? 0.0 : (OP == 1 ? 1e300 : -1e300);
  for (int i = threadIdx.x; i < cols; i += blockDim.x) v = OP == 0 ? v + row[i] : (OP == 1 ? fmin(v, row[i]) : fmax(v, row[i]));
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = OP == 0 ? v + w : (OP == 1 ? fmin(v, w) : fmax(v, w));
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = red[0];
    for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w)
      t = OP == 0 ? t + red[w] : (OP == 1 ? fmin(t, red[w]) : fmax(t, red[w]));
    out[blockIdx.x] = scale * t;
  }
}

__device__ __forceinline__ void chunk_of(int64_t cnt, int64_t& beg, int64_t& end) {
  const int64_t per = (cnt + gridDim.x - 1) / gridDim.x;
  beg = blockIdx.x * per;
  end = beg + per < cnt ? beg + per : cnt;
}

// Gershgorin bounds, stage 1: a warp per row; part[0][b] = min (a_ii - r_i), part[1][b] = max (a_ii + r_i)
// over this CTA's rows.
template <int PL>
__global__ void gershgorin_partial_kernel(const double* A, int64_t n, double* part) {
  __shared__ double lo_s[32], hi_s[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double lo = 1e300, hi = -1e300;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * nw + warp; i < n; i += static_cast<int64_t>(gridDim.x) * nw) {
    double r = 0.0;
    for (int64_t j = lane; j < n; j += 32)
      if (j != i) r += PL == 2 ? hypot(A[(i * n + j) * PL], A[(i * n + j) * PL + 1]) : fabs(A[i * n + j]);
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    lo = fmin(lo, A[(i * n + i) * PL] - r);
    hi = fmax(hi, A[(i * n + i) * PL] + r);
  }
  if (lane == 0) { lo_s[warp] = lo; hi_s[warp] = hi; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < nw; ++w) { lo = fmin(lo, lo_s[w]); hi = fmax(hi, hi_s[w]); }
    lo = fmin(lo, lo_s[0]);
    hi = fmax(hi, hi_s[0]);
    part[blockIdx.x] = lo;
    part[gridDim.x + blockIdx.x] = hi;
  }
}

// SP2 kernels run on RED_CTAS CTAs, each on its chunk of the n x n matrix, and leave per-CTA
// partials (Re tr X, ||X||_F^2) of the matrix they wrote; for Hermitian X, ||X||_F^2 = tr X^2, so
// the next step has both traces without a separate pass over X^2.
template <int PL>
__device__ __forceinline__ void sp2_partials(double tr, double fro, double* red, double* part) {
  tr = block_sum(tr, red);
  fro = block_sum(fro, red);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = tr;
    part[gridDim.x + blockIdx.x] = fro;
  }
}

// X = (emax I - F) / (emax - emin): spectrum mapped into [0, 1], lowest states near 1.
template <int PL>
__global__ void sp2_init_kernel(double* X, const double* F, int64_t n, const double* b, double* part) {
  __shared__ double red[32];
  const double emin = b[0], emax = b[1], inv = 1.0 / fmax(emax - emin, 1e-300);
  int64_t beg, end;
  chunk_of(n * n, beg, end);
  double tr = 0.0, fro = 0.0;
  for (int64_t idx = beg + threadIdx.x; idx < end; idx += blockDim.x) {
    const int64_t i = idx / n, j = idx % n;
    const double re = ((i == j ? emax : 0.0) - F[idx * PL]) * inv;
    X[idx * PL] = re;
    fro += re * re;
    if (i == j) tr += re;
    if (PL == 2) {
      const double im = -F[idx * PL + 1] * inv;
      X[idx * PL + 1] = im;
      fro += im * im;
    }
  }
  sp2_partials<PL>(tr, fro, red, part);
}

// SP2 step (trace correcting): with t1 = tr X and t2 = tr X^2 from the partials `pin` of X,
// X <- X^2 (= T) if that brings the trace closer to N, else 2X - X^2.  tr_out (written by CTA 0)
// receives (t1, t2) for the host's convergence check; `pout` the partials of the new X.
template <int PL>
__global__ void sp2_step_kernel(double* X, const double* T, int64_t n, const double* pin, double* pout,
                                double* tr_out, double N) {
  __shared__ double red[32];
  __shared__ int sq;
  const int np = gridDim.x;  // the partials come from a launch of the same size
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    a += pin[i];
    b += pin[np + i];
  }
  a = block_sum(a, red);
  b = block_sum(b, red);
  if (threadIdx.x == 0) {
    sq = fabs(b - N) < fabs(2.0 * a - b - N) ? 1 : 0;
    if (blockIdx.x == 0) { tr_out[0] = a; tr_out[1] = b; }
  }
  __syncthreads();
  const bool square = sq != 0;
  int64_t beg, end;
  chunk_of(n * n, beg, end);
  double tr = 0.0, fro = 0.0;
  for (int64_t idx = beg + threadIdx.x; idx < end; idx += blockDim.x) {
    const int64_t i = idx / n, j = idx % n;
#pragma unroll
    for (int q = 0; q < PL; ++q) {
      const double x = square ? T[idx * PL + q] : 2.0 * X[idx * PL + q] - T[idx * PL + q];
      X[idx * PL + q] = x;
      fro += x * x;
      if (q == 0 && i == j) tr += x;
    }
  }
  sp2_partials<PL>(tr, fro, red, pout);
}

// Stage 1 of 1/2 Re Tr[P (h + F)]: part[b] = this CTA's share of sum_ij P_ij (h + F)_ji.
template <int PL>
__global__ void energy_partial_kernel(const double* P, const double* h, const double* F, int64_t n, double* part) {
  __shared__ double red[32];
  int64_t beg, end;
  chunk_of(n * n, beg, end);
  double acc = 0.0;
  for (int64_t idx = beg + threadIdx.x; idx < end; idx += blockDim.x) {
    const int64_t i = idx / n, j = idx % n, t = j * n + i;
    acc += P[idx * PL] * (h[t * PL] + F[t * PL]);
    if (PL == 2) acc -= P[idx * PL + 1] * (h[t * PL + 1] + F[t * PL + 1]);
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// Stage 1 of max |A - B|.
template <int PL>
__global__ void maxdiff_partial_kernel(const double* A, const double* B, int64_t cnt, double* part) {
  __shared__ double red[32];
  int64_t beg, end;
  chunk_of(cnt, beg, end);
  double m = 0.0;
  for (int64_t i = beg + threadIdx.x; i < end; i += blockDim.x)
    m = fmax(m, PL == 2 ? hypot(A[2 * i] - B[2 * i], A[2 * i + 1] - B[2 * i + 1]) : fabs(A[i] - B[i]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    part[blockIdx.x] = m;
  }
}

// Time-reversal-even part of a complex n x n matrix in a layout of equal spin blocks of length nb
// alternating alpha / beta ([alpha; beta] X2C AO layout: nb = n/2, src/Utils/KramersPairing.cpp:320;
// [L-alpha; L-beta; S-alpha; S-beta] RKB layout: nb = n/4, :351):
//   out(a, b) = 1/2 (P(a, b) + s_a s_b conj(P(partner a, partner b))),
// partner = the other block of the alpha/beta pair, s = +1 on alpha blocks, -1 on beta blocks.
__global__ void kramers_even_kernel(double* out, const double* P, int64_t n, int64_t nb) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < n * n;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t a = idx / n, b = idx % n;
    const int64_t pa = ((a / nb) ^ 1) * nb + a % nb, pb = ((b / nb) ^ 1) * nb + b % nb;
    const double sg = (((a / nb) % 2 == 0) ? 1.0 : -1.0) * (((b / nb) % 2 == 0) ? 1.0 : -1.0);
    const int64_t q = pa * n + pb;
    out[2 * idx] = 0.5 * (P[2 * idx] + sg * P[2 * q]);
    out[2 * idx + 1] = 0.5 * (P[2 * idx + 1] - sg * P[2 * q + 1]);
  }
}

constexpr int DIIS_MAX = 16;
struct DotArgs {
  const double* v[DIIS_MAX];
  int count;
};

// Stage 1 of <e, v_k>: part[k][b] = this CTA's share.
__global__ void diis_dots_partial_kernel(const double* e, DotArgs a, int64_t cnt, double* part) {
  __shared__ double red[32];
  int64_t beg, end;
  chunk_of(cnt, beg, end);
  for (int k = 0; k < a.count; ++k) {
    double acc = 0.0;
    for (int64_t i = beg + threadIdx.x; i < end; i += blockDim.x) acc += e[i] * a.v[k][i];
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) part[k * gridDim.x + blockIdx.x] = acc;
  }
}

struct CombArgs {
  const double* v[DIIS_MAX];
  double w[DIIS_MAX];
  int count;
};

__global__ void diis_combine_kernel(double* out, CombArgs a, int64_t cnt) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < cnt;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < a.count; ++k) s += a.w[k] * a.v[k][i];
    out[i] = s;
  }
}

// The reference's dense solve (DIIS.cpp:18-48): Gaussian elimination with partial pivoting, false
// when min |pivot| / max |pivot| is not above tol.
bool solve_dense(std::vector<double> m, std::vector<double> rhs, size_t n, double tol, std::vector<double>& x) {
  std::vector<double> piv(n);
  for (size_t k = 0; k < n; ++k) {
    size_t best = k;
    for (size_t i = k + 1; i < n; ++i)
      if (std::fabs(m[i * n + k]) > std::fabs(m[best * n + k])) best = i;
    if (best != k) {
      for (size_t j = 0; j < n; ++j) std::swap(m[k * n + j], m[best * n + j]);
      std::swap(rhs[k], rhs[best]);
    }
    piv[k] = std::fabs(m[k * n + k]);
    if (piv[k] == 0.0) return false;
    for (size_t i = k + 1; i < n; ++i) {
      const double f = m[i * n + k] / m[k * n + k];
      for (size_t j = k; j < n; ++j) m[i * n + j] -= f * m[k * n + j];
      rhs[i] -= f * rhs[k];
    }
  }
  double pmax = piv[0], pmin = piv[0];
  for (double v : piv) { pmax = std::max(pmax, v); pmin = std::min(pmin, v); }
  if (!(pmin > tol * pmax)) return false;
  x.assign(n, 0.0);
  for (size_t ii = n; ii-- > 0;) {
    double sum = rhs[ii];
    for (size_t j = ii + 1; j < n; ++j) sum -= m[ii * n + j] * x[j];
    x[ii] = sum / m[ii * n + ii];
  }
  return true;
}

// Device-resident DIIS history (src/Utils/DIIS.cpp:79-131): slots hold (error, value) pairs; the
// newest-first order and the B matrix are kept on the host.
struct DeviceDiis {
  rr_ri_store* h;  // owns the history buffers; also for host_wait
  int max_vectors = 0;
  int64_t len = 0;
  DevBuf<double>& err;
  DevBuf<double>& val;
  DevBuf<double>& dots;
  std::vector<int> order;  // slot indices, newest first
  std::vector<std::vector<double>> bmat;  // bmat[slot][slot]
  explicit DeviceDiis(rr_ri_store* owner) : h(owner), err(owner->diis_err), val(owner->diis_val), dots(owner->diis_dots) {}
  void init(int maxv, int64_t length) {
    max_vectors = maxv;
    len = length;
    const int slots = std::max(maxv, 1);
    err.ensure(static_cast<size_t>(slots * length));
    val.ensure(static_cast<size_t>(slots * length));
    dots.ensure(DIIS_MAX * (RED_CTAS + 1));
    order.clear();
    bmat.assign(slots, std::vector<double>(slots, 0.0));
  }
  // Stores (e, F) and writes the extrapolated F into out (or copies F when nothing extrapolates).
  void extrapolate(const double* e, const double* F, double* out, cudaStream_t s) {
    if (max_vectors < 2) {
      copy_out(out, F, len, false, s);
      return;
    }
    int slot;
    if (static_cast<int>(order.size()) < max_vectors) {
      slot = static_cast<int>(order.size());
    } else {
      slot = order.back();
      order.pop_back();
    }
    copy_out(err.p + slot * len, e, len, false, s);
    copy_out(val.p + slot * len, F, len, false, s);
    order.insert(order.begin(), slot);
    DotArgs a{};
    a.count = static_cast<int>(order.size());
    for (int k = 0; k < a.count; ++k) a.v[k] = err.p + order[k] * len;
    double* part = dots.p + DIIS_MAX;
    diis_dots_partial_kernel<<<RED_CTAS, 256, 0, s>>>(err.p + slot * len, a, len, part);
    RR_LAUNCH_CHECK();
    reduce_partials_kernel<0><<<a.count, 256, 0, s>>>(part, RED_CTAS, 1.0, dots.p);
    RR_LAUNCH_CHECK();
    std::vector<double> d(a.count);
    RR_CUDA(cudaMemcpyAsync(d.data(), dots.p, sizeof(double) * a.count, cudaMemcpyDeviceToHost, s));
    host_wait(h, s);
    for (int k = 0; k < a.count; ++k) bmat[slot][order[k]] = bmat[order[k]][slot] = d[k];
    const size_t total = order.size();
    for (size_t m = total; m >= 2; --m) {
      double scale = 0.0;
      for (size_t i = 0; i < m; ++i) scale = std::max(scale, bmat[order[i]][order[i]]);
      if (!(scale > 0.0)) break;
      const size_t nn = m + 1;
      std::vector<double> A(nn * nn, 0.0), rhs(nn, 0.0), x;
      for (size_t i = 0; i < m; ++i)
        for (size_t j = 0; j < m; ++j) A[i * nn + j] = bmat[order[i]][order[j]] / scale;
      for (size_t i = 0; i < m; ++i) A[i * nn + m] = A[m * nn + i] = -1.0;
      rhs[m] = -1.0;
      if (!solve_dense(A, rhs, nn, 1e-14, x)) continue;
      CombArgs c{};
      c.count = static_cast<int>(m);
      for (size_t i = 0; i < m; ++i) { c.v[i] = val.p + order[i] * len; c.w[i] = x[i]; }
      diis_combine_kernel<<<blocks_for(len), 256, 0, s>>>(out, c, len);
      RR_LAUNCH_CHECK();
      return;
    }
    copy_out(out, F, len, false, s);
  }
};

// Per-phase device times of an SCF loop (only with profiling on): 0 Fock build, 1 energy + DIIS,
// 2 density step (orthogonal transform, SP2 projector, back-transform, density change).
struct PhaseTimer {
  bool on = false;
  cudaEvent_t ev[4] = {};
  double ms[3] = {0.0, 0.0, 0.0};
  explicit PhaseTimer(bool enable) : on(enable) {
    if (on)
      for (auto& e : ev) RR_CUDA(cudaEventCreate(&e));
  }
  ~PhaseTimer() {
    if (on)
      for (auto& e : ev) cudaEventDestroy(e);
  }
  void mark(int i, cudaStream_t s) {
    if (on) RR_CUDA(cudaEventRecord(ev[i], s));
  }
  // after the stream has passed mark 3
  void accumulate() {
    if (!on) return;
    for (int i = 0; i < 3; ++i) {
      float t = 0.f;
      RR_CUDA(cudaEventElapsedTime(&t, ev[i], ev[i + 1]));
      ms[i] += t;
    }
  }
  // the final FP64 build of a mixed loop (marks 0 and 1 around it, after the stream has passed 1)
  void accumulate_build() {
    if (!on) return;
    float t = 0.f;
    RR_CUDA(cudaEventElapsedTime(&t, ev[0], ev[1]));
    ms[0] += t;
  }
  void store(rr_scf_result* r) const {
    r->build_ms = ms[0];
    r->diis_ms = ms[1];
    r->density_ms = ms[2];
  }
};

// ---- DHF window deflation ----

// F += (b[1] - b[0]) Pi over `cnt` doubles (interleaved complex): the states of the projector Pi move
// up by the width of the spectral interval b, i.e. above every other eigenvalue of F in b.
__global__ void deflate_kernel(double* F, const double* Pi, const double* b, int64_t cnt) {
  const double sigma = b[1] - b[0];
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < cnt;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    F[i] += sigma * Pi[i];
}

// Stage 1 of Re tr(A B) = Re sum_ij A_ij conj(B_ij) for Hermitian A, B (interleaved complex).
__global__ void herm_dot_partial_kernel(const double* A, const double* B, int64_t n2, double* part) {
  __shared__ double red[32];
  int64_t beg, end;
  chunk_of(n2, beg, end);
  double acc = 0.0;
  for (int64_t i = beg + threadIdx.x; i < end; i += blockDim.x) acc += A[2 * i] * B[2 * i] + A[2 * i + 1] * B[2 * i + 1];
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// ---- tight spectral bounds for SP2 (block Krylov Ritz values) ----

// K[:, 0:m] (n rows, row pitch ldk) = deterministic pseudo-random numbers in [-1, 1) (splitmix64).
template <int PL>
__global__ void krylov_start_kernel(double* K, int64_t n, int ldk, int m) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < n * m * PL;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t row = idx / (m * PL), c = idx % (m * PL);
    uint64_t z = static_cast<uint64_t>(idx) * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    K[row * ldk * PL + c] = static_cast<double>(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
  }
}

// Columns c0 .. c0 + gridDim.x - 1 of K scaled to unit 2-norm (one CTA per column).
template <int PL>
__global__ void normalize_cols_kernel(double* K, int64_t n, int ldk, int c0) {
  __shared__ double red[32];
  __shared__ double scale;
  const int c = c0 + blockIdx.x;
  double s2 = 0.0;
  for (int64_t r = threadIdx.x; r < n; r += blockDim.x)
#pragma unroll
    for (int q = 0; q < PL; ++q) {
      const double v = K[(r * ldk + c) * PL + q];
      s2 += v * v;
    }
  s2 = block_sum(s2, red);
  if (threadIdx.x == 0) scale = s2 > 0.0 ? 1.0 / sqrt(s2) : 0.0;
  __syncthreads();
  for (int64_t r = threadIdx.x; r < n; r += blockDim.x)
#pragma unroll
    for (int q = 0; q < PL; ++q) K[(r * ldk + c) * PL + q] *= scale;
}

// b = [lo, hi] (the Gershgorin interval on entry) narrowed to the Ritz interval widened by 10% of
// its spread on both sides, when the small eigenproblem succeeded.
__global__ void ritz_bounds_kernel(const double* w, int k, const int* info, double* b) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double lo = w[0], hi = w[k - 1], spread = hi - lo;
  if (*info != 0 || !(spread >= 0.0) || !isfinite(lo) || !isfinite(hi)) return;
  const double m = 0.1 * spread + 1e-12 * fmax(fabs(lo), fabs(hi));
  const double nlo = fmax(b[0], lo - m), nhi = fmin(b[1], hi + m);
  if (nhi > nlo) { b[0] = nlo; b[1] = nhi; }
}

}  // namespace

bool diis_solve(const std::vector<double>& m, const std::vector<double>& rhs, size_t n, double tol,
                std::vector<double>& x) {
  return solve_dense(m, rhs, n, tol, x);
}

// Narrows the SP2 spectral interval b (device, [lo, hi], Gershgorin on entry) of the Hermitian n x n
// F with the Ritz values of F on the block Krylov space [V, F V, F^2 V, F^3 V] (V: 8 fixed
// pseudo-random vectors), widened by 10% of their spread: a generalized 32 x 32 eigenproblem
// (K^dagger F K) y = theta (K^dagger K) y on the device (cuSOLVER).  Small matrices keep b.
void ritz_bounds(rr_ri_store* h, const double* F, int64_t n, bool cplx, double* b, cudaStream_t s) {
  constexpr int m = 8, q = 4, k = m * q;
  if (n < 4 * k) return;
  const int PL = cplx ? 2 : 1;
  double *K, *FK, *T, *M, *w;
  Arena ar(&h->solver_a);
  ar.request(&K, n * k * PL);
  ar.request(&FK, n * k * PL);
  ar.request(&T, k * k * PL);
  ar.request(&M, k * k * PL);
  ar.request(&w, k);
  ar.commit();
  if (cplx) krylov_start_kernel<2><<<blocks_for(n * m * 2), 256, 0, s>>>(K, n, k, m);
  else krylov_start_kernel<1><<<blocks_for(n * m), 256, 0, s>>>(K, n, k, m);
  RR_LAUNCH_CHECK();
  for (int j = 0; j < q; ++j) {
    if (j > 0) {
      GemmDesc g;
      g.cplx = cplx;
      g.M = n; g.N = m; g.K = n;
      g.A = F; g.lda = n; g.B = K + (j - 1) * m * PL; g.ldb = k; g.C = K + j * m * PL; g.ldc = k;
      gemm(g, s, h->work.p, static_cast<int64_t>(h->work.n));
    }
    if (cplx) normalize_cols_kernel<2><<<m, 256, 0, s>>>(K, n, k, j * m);
    else normalize_cols_kernel<1><<<m, 256, 0, s>>>(K, n, k, j * m);
    RR_LAUNCH_CHECK();
  }
  GemmDesc f;
  f.cplx = cplx;
  f.M = n; f.N = k; f.K = n; f.A = F; f.lda = n; f.B = K; f.ldb = k; f.C = FK; f.ldc = k;
  gemm(f, s, h->work.p, static_cast<int64_t>(h->work.n));
  GemmDesc t;
  t.cplx = cplx;
  t.M = k; t.N = k; t.K = n; t.A = K; t.lda = k; t.opA = Op::T; t.conjA = cplx; t.B = FK; t.ldb = k; t.C = T; t.ldc = k;
  gemm(t, s, h->work.p, static_cast<int64_t>(h->work.n));
  t.B = K; t.C = M;
  t.mirror = 1;
  gemm(t, s, h->work.p, static_cast<int64_t>(h->work.n));
  auto& c = h->ctx;
  RR_SOLVER(cusolverDnSetStream(c.solver, s));
  c.solver_info.ensure(1);
  int lwork = 0;
  if (cplx) {
    auto* tz = reinterpret_cast<cuDoubleComplex*>(T);
    auto* mz = reinterpret_cast<cuDoubleComplex*>(M);
    RR_SOLVER(cusolverDnZhegvd_bufferSize(c.solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_NOVECTOR,
                                          CUBLAS_FILL_MODE_UPPER, k, tz, k, mz, k, w, &lwork));
    c.solver_work.ensure(2 * static_cast<size_t>(lwork) + 2);
    RR_SOLVER(cusolverDnZhegvd(c.solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_NOVECTOR, CUBLAS_FILL_MODE_UPPER, k,
                               tz, k, mz, k, w, reinterpret_cast<cuDoubleComplex*>(c.solver_work.p), lwork,
                               c.solver_info.p));
  } else {
    RR_SOLVER(cusolverDnDsygvd_bufferSize(c.solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_NOVECTOR,
                                          CUBLAS_FILL_MODE_UPPER, k, T, k, M, k, w, &lwork));
    c.solver_work.ensure(static_cast<size_t>(lwork) + 1);
    RR_SOLVER(cusolverDnDsygvd(c.solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_NOVECTOR, CUBLAS_FILL_MODE_UPPER, k, T,
                               k, M, k, w, c.solver_work.p, lwork, c.solver_info.p));
  }
  ritz_bounds_kernel<<<1, 32, 0, s>>>(w, k, c.solver_info.p, b);
  RR_LAUNCH_CHECK();
}

// SP2 purification: projector (n x n, into Pi) onto the lowest `nocc` eigenvectors of the symmetric
// (Hermitian when cplx, interleaved) F (n x n).  T is scratch (n x n).  Host checks every 4 steps;
// at most 120 steps.
void sp2_projector(rr_ri_store* h, const double* F, int64_t n, int64_t nocc, double* Pi, double* T, double* scal,
                   cudaStream_t s, bool cplx) {
  const int PL = cplx ? 2 : 1;
  h->work.ensure(static_cast<size_t>(std::max<int64_t>(static_cast<int64_t>(h->work.n), 8 * n * n * PL + 6 * RED_CTAS)));
  double* part = h->work.p;  // Gershgorin partials, then the SP2 trace partials
  const int gcta = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(RED_CTAS, (n + 7) / 8)));
  if (cplx) gershgorin_partial_kernel<2><<<gcta, 256, 0, s>>>(F, n, part);
  else gershgorin_partial_kernel<1><<<gcta, 256, 0, s>>>(F, n, part);
  RR_LAUNCH_CHECK();
  reduce_partials_kernel<1><<<1, 256, 0, s>>>(part, gcta, 1.0, scal);
  RR_LAUNCH_CHECK();
  reduce_partials_kernel<2><<<1, 256, 0, s>>>(part + gcta, gcta, 1.0, scal + 1);
  RR_LAUNCH_CHECK();
  // Gershgorin interval kept in scal[4..5]; the Ritz interval (tighter: fewer SP2 steps) is tried first
  RR_CUDA(cudaMemcpyAsync(scal + 4, scal, 2 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  ritz_bounds(h, F, n, cplx, scal, s);
  // ping-pong partials of X after the Gershgorin partials (the GEMM's split-K scratch follows them)
  double* sp_part[2] = {part + 2 * RED_CTAS, part + 4 * RED_CTAS};
  auto init = [&] {
    if (cplx) sp2_init_kernel<2><<<RED_CTAS, 256, 0, s>>>(Pi, F, n, scal, sp_part[0]);
    else sp2_init_kernel<1><<<RED_CTAS, 256, 0, s>>>(Pi, F, n, scal, sp_part[0]);
    RR_LAUNCH_CHECK();
  };
  init();
  GemmDesc g;
  g.cplx = cplx;
  g.M = n; g.N = n; g.K = n;
  g.A = Pi; g.lda = n; g.B = Pi; g.ldb = n; g.C = T; g.ldc = n;
  g.mirror = 1;  // X is Hermitian, so is X^2: upper tiles, the rest mirrored
  const double N = static_cast<double>(nocc);
  double* gw = part + 6 * RED_CTAS;  // split-K scratch of the X^2 products
  const int64_t gcap = static_cast<int64_t>(h->work.n) - 6 * RED_CTAS;
  bool gershgorin = false;
  for (int it = 0, step = 0; step < 120; ++it, ++step) {
    gemm(g, s, gw, gcap);
    if (cplx)
      sp2_step_kernel<2><<<RED_CTAS, 256, 0, s>>>(Pi, T, n, sp_part[it & 1], sp_part[(it + 1) & 1], scal + 2, N);
    else
      sp2_step_kernel<1><<<RED_CTAS, 256, 0, s>>>(Pi, T, n, sp_part[it & 1], sp_part[(it + 1) & 1], scal + 2, N);
    RR_LAUNCH_CHECK();
    if (it % 4 == 3) {
      double tr[2];
      RR_CUDA(cudaMemcpyAsync(tr, scal + 2, sizeof(tr), cudaMemcpyDeviceToHost, s));
      host_wait(h, s);
      // idempotency measure of the pre-update X: |tr X - tr X^2| (sum of lambda (1 - lambda))
      if (std::fabs(tr[0] - tr[1]) < 1e-11 * std::max<double>(1.0, N) && std::fabs(tr[0] - N) < 1e-6) return;
      // With every eigenvalue of X in [0, 1], tr X^2 <= tr X; otherwise the Ritz interval missed part
      // of the spectrum: start again from the Gershgorin interval.
      if (!gershgorin && (tr[1] > tr[0] + 1e-9 * std::max<double>(1.0, N) || step + 1 >= 60)) {
        gershgorin = true;
        RR_CUDA(cudaMemcpyAsync(scal, scal + 4, 2 * sizeof(double), cudaMemcpyDeviceToDevice, s));
        init();
        it = -1;
        step = -1;
      }
    }
  }
  throw Error(RR_ERR_SOLVER, "SCF: density purification did not converge (no gap at the Fermi level?)");
}

// Orbital energies, coefficients and Fock matrix of an SCF loop's last iteration, as the reference's
// SCF results carry them (src/NON_REL/NonRelHartreeFock.h:28-38, src/X2C_DHF/X2C_HF.h:28-37,
// src/C4_DHF/C4_DHF.h:28-36; filled at NonRelHartreeFock.cpp:146-151): w and U from
// X^dagger F X = U diag(w) U^dagger (cuSOLVER syevd / heevd on the device, w ascending), C = X U, and
// F itself.  Only the outputs whose pointers the caller set are formed.
void scf_result_outputs(rr_ri_store* h, const double* F, const double* Xd, int64_t n, int64_t n_eff, bool cplx,
                        const rr_scf_result* res, bool host, cudaStream_t s) {
  const int PL = cplx ? 2 : 1;
  if (res->fock_matrix) copy_out(res->fock_matrix, F, n * n * PL, host, s);
  if (!res->orbital_energies && !res->c_matrix) return;
  double *FX, *A, *w, *C;
  Arena ar(&h->solver_a);
  ar.request(&FX, n * n_eff * PL);
  ar.request(&A, n_eff * n_eff * PL);
  ar.request(&w, n_eff);
  ar.request(&C, n * n_eff * PL);
  ar.commit();
  auto wk = [h] { return h->work.p; };
  auto wcap = [h] { return static_cast<int64_t>(h->work.n); };
  GemmDesc a;
  a.cplx = cplx;
  a.M = n; a.N = n_eff; a.K = n; a.A = F; a.lda = n; a.B = Xd; a.ldb = n_eff; a.C = FX; a.ldc = n_eff;
  gemm(a, s, wk(), wcap());
  a.M = n_eff; a.N = n_eff; a.K = n; a.A = Xd; a.lda = n_eff; a.opA = Op::T; a.conjA = cplx; a.B = FX; a.ldb = n_eff;
  a.C = A; a.ldc = n_eff;
  a.mirror = 1;  // X^dagger F X is Hermitian
  gemm(a, s, wk(), wcap());
  // row j of A: eigenvector j (conjugated for the complex solver, which sees the row-major matrix as
  // its transpose)
  if (cplx) eigh_herm(h, A, n_eff, w, s);
  else eigh_sym(h, A, n_eff, w, s);
  int info = 0;
  RR_CUDA(cudaMemcpyAsync(&info, h->ctx.solver_info.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  host_wait(h, s);
  RR_REQUIRE(info == 0, RR_ERR_SOLVER,
             "SCF result: the eigensolver of X^dagger F X did not converge (info " + std::to_string(info) + ")");
  if (res->orbital_energies) copy_out(res->orbital_energies, w, n_eff, host, s);
  if (res->c_matrix) {
    GemmDesc c;  // C = X U, U = A^dagger (complex) or A^T (real)
    c.cplx = cplx;
    c.M = n; c.N = n_eff; c.K = n_eff; c.A = Xd; c.lda = n_eff; c.B = A; c.ldb = n_eff; c.opB = Op::T;
    c.conjB = cplx; c.C = C; c.ldc = n_eff;
    gemm(c, s, wk(), wcap());
    copy_out(res->c_matrix, C, n * n_eff * PL, host, s);
  }
}

void scf_nonrel(rr_ri_store* h, const double* hc, const double* X, int64_t n_eff, const double* S, const double* P0,
                int n_electrons, const rr_scf_opts* so, rr_scf_result* res, double* P_out, double* hist,
                const rr_opts* o) {
  RR_REQUIRE(h->ntens == 1, RR_ERR_STATE, "rr_scf_run_nonrel: handle holds a 4-component store");
  RR_REQUIRE(n_electrons > 0 && n_electrons % 2 == 0, RR_ERR_ARG,
             "nonRelDensityMatrix: n_electrons must be a positive even number (closed-shell restricted Hartree-Fock)");
  const int64_t n = h->n, n2 = n * n, nocc = n_electrons / 2;
  RR_REQUIRE(nocc <= n_eff, RR_ERR_ARG, "nonRelDensityMatrix: n_electrons/2 exceeds the number of available spatial orbitals");
  const bool host = !o || o->mem == RR_MEM_HOST;
  cudaStream_t s = call_stream(h, o);
  const auto t_start = std::chrono::steady_clock::now();
  const int64_t pitch = round_up(std::max<int64_t>(n2, 2), 32);
  Arena ar(&h->scf_buf);
  double *hd, *Xd, *Sd, *P, *Pn, *F, *J, *K, *Fs, *e, *PS, *SP, *tmp, *Fo, *Pi, *T2, *Ct, *scal, *red;
  ar.request(&hd, n2);
  ar.request(&Xd, n * n_eff);
  ar.request(&Sd, n2);
  ar.request(&P, pitch);
  ar.request(&Pn, pitch);
  ar.request(&F, n2);
  ar.request(&J, n2);
  ar.request(&K, n2);
  ar.request(&Fs, n2);
  ar.request(&e, n2);
  ar.request(&PS, n2);
  ar.request(&SP, n2);
  ar.request(&tmp, std::max(n2, n * n_eff));
  ar.request(&Fo, n_eff * n_eff);
  ar.request(&Pi, n_eff * n_eff);
  ar.request(&T2, n_eff * n_eff);
  ar.request(&Ct, nocc * n);
  ar.request(&scal, 64);
  ar.request(&red, RED_CTAS);
  ar.commit();
  copy_in(hd, hc, n2, host, s);
  copy_in(Xd, X, n * n_eff, host, s);
  copy_in(Sd, S, n2, host, s);
  copy_in_padded(P, pitch, P0, n2, host, s);
  RR_CUDA(cudaMemsetAsync(Pn + n2, 0, sizeof(double) * (pitch - n2), s));
  // Mixed precision: after the first (FP64, drop-in) build, a full split-BF16 exchange, then builds
  // that add the split-BF16 exchange of the change of c_t (its error shrinks with the density
  // change), re-seeded once by an FP64 exchange when |dE| < mixed_switch; once converged, one FP64
  // build of the newest density gives the reported energy.
  const bool mixed = so->precision == RR_PREC_MIXED;
  bool reseed = false, reseeded = false;
  h->inc_r = -1;
  DeviceDiis diis(h);
  const bool use_diis = so->diis_size >= 2;
  diis.init(use_diis ? so->diis_size : 0, n2);
  RR_REQUIRE(so->diis_size <= DIIS_MAX, RR_ERR_ARG, "rr_scf_run_nonrel: diis_size too large");
  h->work.ensure(static_cast<size_t>(std::max<int64_t>(static_cast<int64_t>(h->work.n), 8 * n2)));
  GemmDesc g;
  g.M = n; g.N = n; g.K = n; g.lda = n; g.ldb = n; g.ldc = n;
  double prev = 0.0;
  int64_t it = 0, n_mixed = 0, n_fp64 = 0;
  bool converged = false;
  PhaseTimer pt(h->profiling);
  for (it = 1; it <= so->max_iterations; ++it) {
    pt.mark(0, s);
    // ---- Fock matrix of the current density ----
    if (it == 1) {
      rr_opts od{};
      od.mem = RR_MEM_DEVICE;
      od.stream = s;
      od.sync = 0;
      fock_nonrel(h, hd, P, Sd, Xd, n_eff, F, &od);
      ++n_fp64;
    } else if (mixed) {
      // the exchange accumulates in h->inc_k: a full split-BF16 exchange first, then the split-BF16
      // exchange of the change of c_t (or, once, an FP64 re-seed); J stays FP64
      h->inc_k.ensure(static_cast<size_t>(n2));
      if (reseed) {
        exchange_nonrel(h, Ct, n, false, nocc, h->inc_k.p, s, P, J);
        ++n_fp64;
      } else {
        mixed_prepare(h->mixed[0], h->B[0].p, h->pitch[0], n, h->naux, s);
        const bool incr = h->inc_r == nocc && h->inc_ld == n;
        ExFlavours fl;
        fl.nf = 1;
        fl.fs[0] = n;
        mixed_exchange_general(h->mixed, h->mscr, fl, h->naux, Ct, incr ? h->inc_ct.p : nullptr, n, nocc, false,
                               h->inc_k.p, n, incr, h->status.p, s);
        coulomb_after_ht(h, P, Ct, 0, J, nullptr, 0, s);
        ++n_mixed;
      }
      reseed = false;
      h->inc_ct.ensure(static_cast<size_t>(std::max<int64_t>(nocc * n, 1)));
      RR_CUDA(cudaMemcpyAsync(h->inc_ct.p, Ct, sizeof(double) * nocc * n, cudaMemcpyDeviceToDevice, s));
      h->inc_r = nocc;
      h->inc_ld = n;
      coulomb_join(h, s);
      fock_combine(F, hd, J, h->inc_k.p, n2, s);
    } else {
      exchange_nonrel(h, Ct, n, false, nocc, K, s, P, J);
      coulomb_join(h, s);
      fock_combine(F, hd, J, K, n2, s);
      ++n_fp64;
    }
    pt.mark(1, s);
    // ---- energy with the un-extrapolated F ----
    energy_partial_kernel<1><<<RED_CTAS, 256, 0, s>>>(P, hd, F, n, red);
    RR_LAUNCH_CHECK();
    reduce_partials_kernel<0><<<1, 256, 0, s>>>(red, RED_CTAS, 0.5, scal);
    RR_LAUNCH_CHECK();
    // ---- DIIS on e = F P S - S P F ----
    if (use_diis) {
      g.A = P; g.B = Sd; g.C = PS; g.alpha = 1.0; g.beta = 0.0;
      gemm(g, s, h->work.p, static_cast<int64_t>(h->work.n));
      g.A = Sd; g.B = P; g.C = SP;
      gemm(g, s, h->work.p, static_cast<int64_t>(h->work.n));
      g.A = F; g.B = PS; g.C = e;
      gemm(g, s, h->work.p, static_cast<int64_t>(h->work.n));
      g.A = SP; g.B = F; g.C = e; g.alpha = -1.0; g.beta = 1.0;
      gemm(g, s, h->work.p, static_cast<int64_t>(h->work.n));
      diis.extrapolate(e, F, Fs, s);
    } else {
      copy_out(Fs, F, n2, false, s);
    }
    pt.mark(2, s);
    // ---- F_ortho = X^T F_scf X, aufbau projector, new orbitals and density ----
    GemmDesc a;
    a.M = n; a.N = n_eff; a.K = n; a.A = Fs; a.lda = n; a.B = Xd; a.ldb = n_eff; a.C = tmp; a.ldc = n_eff;
    gemm(a, s, h->work.p, static_cast<int64_t>(h->work.n));
    a.M = n_eff; a.N = n_eff; a.K = n; a.A = Xd; a.lda = n_eff; a.opA = Op::T; a.B = tmp; a.ldb = n_eff; a.C = Fo;
    a.ldc = n_eff;
    a.mirror = 1;  // X^T F X is symmetric
    gemm(a, s, h->work.p, static_cast<int64_t>(h->work.n));
    sp2_projector(h, Fo, n_eff, nocc, Pi, T2, scal + 8, s, false);
    projector_ct(h, Pi, nullptr, Xd, n, n_eff, nocc, false, Ct, s);
    GemmDesc dp;
    dp.M = n; dp.N = n; dp.K = nocc; dp.A = Ct; dp.lda = n; dp.opA = Op::T; dp.B = Ct; dp.ldb = n; dp.C = Pn; dp.ldc = n;
    dp.alpha = 2.0;
    dp.mirror = 1;  // 2 C C^T is symmetric
    gemm(dp, s, h->work.p, static_cast<int64_t>(h->work.n));
    maxdiff_partial_kernel<1><<<RED_CTAS, 256, 0, s>>>(Pn, P, n2, red);
    RR_LAUNCH_CHECK();
    reduce_partials_kernel<2><<<1, 256, 0, s>>>(red, RED_CTAS, 1.0, scal + 1);
    RR_LAUNCH_CHECK();
    pt.mark(3, s);
    double hv[2];
    RR_CUDA(cudaMemcpyAsync(hv, scal, sizeof(hv), cudaMemcpyDeviceToHost, s));
    host_wait(h, s);
    pt.accumulate();
    const double energy = hv[0], dP = hv[1], dE = std::fabs(energy - prev);
    if (hist) hist[it - 1] = energy;
    res->electronic_energy = energy;
    const bool conv = it > 1 && (dP < so->density_tolerance || dE < so->energy_tolerance);
    prev = energy;
    const bool mixing_on = !use_diis && so->mixing > 0.0 && so->mixing != 1.0;
    if (conv) {
      if (mixed) {
        // last iteration in FP64: the FP64 Fock matrix of the newest density and its energy
        // Unless the caller asked for the Fock matrix or orbitals, only the FP64 energy is formed: J and
        // the half-transform give 1/2 Tr[D (h + F)] = Tr[D h] + E_J - E_K without the exchange SYRK.
        if (mixing_on) axpby(Pn, P, 1.0 - so->mixing, so->mixing, n2, s);
        std::swap(P, Pn);
        // (with linear mixing the density is not 2 Ct^T Ct, so the full build gives its energy)
        const bool full_fock = res->fock_matrix || res->c_matrix || res->orbital_energies || mixing_on;
        pt.mark(0, s);
        double ev = 0.0;
        if (full_fock) {
          exchange_nonrel(h, Ct, n, false, nocc, K, s, P, J);
          coulomb_join(h, s);
          fock_combine(F, hd, J, K, n2, s);
          pt.mark(1, s);
          energy_partial_kernel<1><<<RED_CTAS, 256, 0, s>>>(P, hd, F, n, red);
          RR_LAUNCH_CHECK();
          reduce_partials_kernel<0><<<1, 256, 0, s>>>(red, RED_CTAS, 0.5, scal);
          RR_LAUNCH_CHECK();
          RR_CUDA(cudaMemcpyAsync(&ev, scal, sizeof(double), cudaMemcpyDeviceToHost, s));
        } else {
          energy_nonrel(h, Ct, nocc, P, J, scal + 24, s);
          pt.mark(1, s);
          // Tr[D h] = 1/2 sum_ij D_ij (h + h)_ji
          energy_partial_kernel<1><<<RED_CTAS, 256, 0, s>>>(P, hd, hd, n, red);
          RR_LAUNCH_CHECK();
          reduce_partials_kernel<0><<<1, 256, 0, s>>>(red, RED_CTAS, 0.5, scal + 26);
          RR_LAUNCH_CHECK();
          double e3[3];
          RR_CUDA(cudaMemcpyAsync(e3, scal + 24, sizeof(e3), cudaMemcpyDeviceToHost, s));
          host_wait(h, s);
          ev = e3[2] + e3[0] - e3[1];
        }
        ++n_fp64;
        host_wait(h, s);
        pt.accumulate_build();
        res->electronic_energy = ev;
        if (it < so->max_iterations) {
          ++it;
          if (hist) hist[it - 1] = ev;
        }
      }
      converged = true;
      break;
    }
    if (mixed && !reseeded && so->mixed_switch > 0.0 && it > 1 && dE < so->mixed_switch) reseed = reseeded = true;
    if (mixing_on) {
      // linear mixing: only the density of the next build changes (NonRelHartreeFock.cpp:185-195)
      axpby(Pn, P, 1.0 - so->mixing, so->mixing, n2, s);
    }
    std::swap(P, Pn);
  }
  if (it > so->max_iterations) it = so->max_iterations;
  // the converged mixed loop's last Fock matrix is the FP64 build of the final density (no DIIS step
  // follows it); otherwise the last iteration's DIIS-extrapolated F, as the reference reports
  scf_result_outputs(h, mixed && converged ? F : Fs, Xd, n, n_eff, false, res, host, s);
  check_status(h, s);
  copy_out(P_out, P, n2, host, s);
  host_wait(h, s);
  res->iterations = it;
  res->converged = converged ? 1 : 0;
  res->mixed_iterations = n_mixed;
  res->fp64_iterations = n_fp64;
  res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  pt.store(res);
}

// X2C-HF (kind 0) and 4c-DHF (kind 1) SCF loops on the device (X2C_HF.cpp:43-138,
// C4_DHF.cpp:45-142).  Matrices are complex interleaved.  The Fock build is the drop-in one
// (x2cFockMatrix / rkbFockMatrix, occupied recovery from the density included); the new density is
// X Pi X^dagger with Pi from SP2 (X2C: lowest n_e states; DHF: the n_e states above the n/2
// negative-energy ones, as the difference of two projectors).
void scf_rel(rr_ri_store* h, int kind, const double* hc, const double* v_total, int64_t n, const double* X,
             int64_t n_eff, const double* S, const double* P0, int n_electrons, const rr_scf_opts* so,
             rr_scf_result* res, double* P_out, double* hist, const rr_opts* o) {
  const bool dhf = kind == 1;
  const int64_t n2 = n * n, c2 = 2 * n2, ce = 2 * n * n_eff, ee = 2 * n_eff * n_eff;
  const int64_t nlo = dhf ? n / 2 : 0;  // states below the occupied window
  RR_REQUIRE(n_electrons > 0 && nlo + n_electrons <= n_eff, RR_ERR_ARG,
             dhf ? "rkbDensityMatrix: n_electrons must be a positive number of spinors that fits within the "
                   "positive-energy half of the RKB basis"
                 : "x2cDensityMatrix: n_electrons must be a positive number of spinors that fits within the basis");
  const bool host = !o || o->mem == RR_MEM_HOST;
  cudaStream_t s = call_stream(h, o);
  const auto t_start = std::chrono::steady_clock::now();
  const int64_t nu = dhf ? 2 * h->n + 2 * h->ns : 0;
  Arena ar(&h->scf_buf);
  double *hd, *Xd, *Sd, *vd = nullptr, *P, *Pn, *F, *Fs, *e, *PS, *SP, *tmp, *Fo, *Pi, *Pi2, *T2, *scal, *red;
  ar.request(&hd, c2);
  ar.request(&Xd, ce);
  ar.request(&Sd, c2);
  if (dhf) ar.request(&vd, 2 * nu * n);
  ar.request(&P, c2);
  ar.request(&Pn, c2);
  ar.request(&F, c2);
  ar.request(&Fs, c2);
  ar.request(&e, c2);
  ar.request(&PS, c2);
  ar.request(&SP, c2);
  ar.request(&tmp, std::max(c2, ce));
  ar.request(&Fo, ee);
  ar.request(&Pi, ee);
  ar.request(&Pi2, dhf ? ee : 1);
  ar.request(&T2, ee);
  ar.request(&scal, 64);
  ar.request(&red, RED_CTAS);
  ar.commit();
  copy_in(hd, hc, c2, host, s);
  copy_in(Xd, X, ce, host, s);
  copy_in(Sd, S, c2, host, s);
  if (dhf) copy_in(vd, v_total, 2 * nu * n, host, s);
  const bool restrict_active = so->kramers_restricted && n_electrons % 2 == 0;
  const int64_t nb = dhf ? n / 4 : n / 2;
  if (restrict_active) {
    copy_in(Pn, P0, c2, host, s);
    kramers_even_kernel<<<blocks_for(n2), 256, 0, s>>>(P, Pn, n, nb);
    RR_LAUNCH_CHECK();
  } else {
    copy_in(P, P0, c2, host, s);
  }
  DeviceDiis diis(h);
  const bool use_diis = so->diis_size >= 2;
  RR_REQUIRE(so->diis_size <= DIIS_MAX, RR_ERR_ARG, "SCF: diis_size too large");
  diis.init(use_diis ? so->diis_size : 0, c2);
  h->work.ensure(static_cast<size_t>(std::max<int64_t>(static_cast<int64_t>(h->work.n), 8 * c2)));
  // The Fock build may grow h->work (split-K partials of the exchange), so every product below
  // takes the buffer as it is at its own call.
  auto wk = [h] { return h->work.p; };
  auto wcap = [h] { return static_cast<int64_t>(h->work.n); };
  GemmDesc g;  // n x n complex products
  g.cplx = true;
  g.M = n; g.N = n; g.K = n; g.lda = n; g.ldb = n; g.ldc = n;
  rr_opts od{};
  od.mem = RR_MEM_DEVICE;
  od.stream = s;
  double prev = 0.0;
  int64_t it = 0, n_mixed = 0, n_fp64 = 0;
  bool converged = false;
  // Mixed precision: the first build is a full split-BF16 one, every later build adds the split-BF16
  // exchange of the change of c_t (its error shrinks with the density change), optionally re-seeded
  // once by an FP64 build when |dE| < mixed_switch; once converged, the last iteration is an FP64
  // build of the final density whose energy is reported.
  bool mixed = so->precision == RR_PREC_MIXED, reseed = false, reseeded = false;
  h->inc_r = -1;
  // After the first iteration the density is X Pi X^dagger (Kramers-projected) with Pi the SP2
  // (window) projector, so the builds take the occupied spinors from Pi; linear mixing makes the
  // density non-idempotent and keeps the recovery from P.
  const bool mixing_on = !use_diis && so->mixing > 0.0 && so->mixing != 1.0;
  bool have_proj = false;
  auto build = [&](const RelBuild* rb) {
    const double* pj = have_proj ? Pi : nullptr;
    const int64_t pr = have_proj ? n_electrons : 0;
    if (dhf) fock_rkb(h, hd, vd, n, Sd, Xd, n_eff, P, F, &od, rb, pj, pr);
    else fock_x2c(h, hd, P, Sd, Xd, n_eff, F, &od, rb, pj, pr);
  };
  auto energy_of_f = [&] {
    energy_partial_kernel<2><<<RED_CTAS, 256, 0, s>>>(P, hd, F, n, red);
    RR_LAUNCH_CHECK();
    reduce_partials_kernel<0><<<1, 256, 0, s>>>(red, RED_CTAS, 0.5, scal);
    RR_LAUNCH_CHECK();
  };
  PhaseTimer pt(h->profiling);
  for (it = 1; it <= so->max_iterations; ++it) {
    pt.mark(0, s);
    if (mixed) {
      RelBuild rb;
      rb.mixed = !reseed;
      rb.incremental = it > 1;
      build(&rb);
      if (reseed) ++n_fp64;
      else ++n_mixed;
      reseed = false;
    } else {
      build(nullptr);
      ++n_fp64;
    }
    pt.mark(1, s);
    energy_of_f();
    if (use_diis) {
      g.A = P; g.B = Sd; g.C = PS; g.alpha = 1.0; g.beta = 0.0;
      gemm(g, s, wk(), wcap());
      g.A = Sd; g.B = P; g.C = SP;
      gemm(g, s, wk(), wcap());
      g.A = F; g.B = PS; g.C = e;
      gemm(g, s, wk(), wcap());
      g.A = SP; g.B = F; g.C = e; g.alpha = -1.0; g.beta = 1.0;
      gemm(g, s, wk(), wcap());
      g.alpha = 1.0; g.beta = 0.0;
      diis.extrapolate(e, F, Fs, s);
    } else {
      copy_out(Fs, F, c2, false, s);
    }
    pt.mark(2, s);
    // F_ortho = X^dagger F_scf X
    GemmDesc a;
    a.cplx = true;
    a.M = n; a.N = n_eff; a.K = n; a.A = Fs; a.lda = n; a.B = Xd; a.ldb = n_eff; a.C = tmp; a.ldc = n_eff;
    gemm(a, s, wk(), wcap());
    a.M = n_eff; a.N = n_eff; a.K = n; a.A = Xd; a.lda = n_eff; a.opA = Op::T; a.conjA = true; a.B = tmp;
    a.ldb = n_eff; a.C = Fo; a.ldc = n_eff;
    a.mirror = 1;  // X^dagger F X is Hermitian
    gemm(a, s, wk(), wcap());
    // window projector in the orthonormal basis
    if (nlo > 0) {
      // DHF: the negative-energy projector first (a wide gap: few SP2 steps), then those states are
      // moved above the whole spectrum (F' = F + sigma Pi_neg, sigma = width of the interval SP2
      // used) and the window is the lowest n_electrons states of F', whose spectral interval no
      // longer spans the negative-energy continuum.  tr(Pi Pi_neg) ~ 0 confirms that no shifted
      // state stayed below the window; otherwise the window is Pi_{nlo + n_e}(F) - Pi_{nlo}(F).
      sp2_projector(h, Fo, n_eff, nlo, Pi2, T2, scal + 8, s, true);
      RR_CUDA(cudaMemcpyAsync(tmp, Fo, sizeof(double) * ee, cudaMemcpyDeviceToDevice, s));
      deflate_kernel<<<blocks_for(ee), 256, 0, s>>>(Fo, Pi2, scal + 8, ee);
      RR_LAUNCH_CHECK();
      sp2_projector(h, Fo, n_eff, n_electrons, Pi, T2, scal + 8, s, true);
      herm_dot_partial_kernel<<<RED_CTAS, 256, 0, s>>>(Pi, Pi2, n_eff * n_eff, red);
      RR_LAUNCH_CHECK();
      reduce_partials_kernel<0><<<1, 256, 0, s>>>(red, RED_CTAS, 1.0, scal + 16);
      RR_LAUNCH_CHECK();
      double leak = 0.0;
      RR_CUDA(cudaMemcpyAsync(&leak, scal + 16, sizeof(double), cudaMemcpyDeviceToHost, s));
      host_wait(h, s);
      if (!(std::fabs(leak) < 1e-6)) {
        sp2_projector(h, tmp, n_eff, nlo + n_electrons, Pi, T2, scal + 8, s, true);
        axpby(Pi, Pi2, -1.0, 1.0, ee, s);
      }
    } else {
      sp2_projector(h, Fo, n_eff, nlo + n_electrons, Pi, T2, scal + 8, s, true);
    }
    // P_new = X Pi X^dagger (Kramers-projected)
    GemmDesc b;
    b.cplx = true;
    b.M = n; b.N = n_eff; b.K = n_eff; b.A = Xd; b.lda = n_eff; b.B = Pi; b.ldb = n_eff; b.C = tmp; b.ldc = n_eff;
    gemm(b, s, wk(), wcap());
    b.M = n; b.N = n; b.K = n_eff; b.A = tmp; b.lda = n_eff; b.B = Xd; b.ldb = n_eff; b.opB = Op::T; b.conjB = true;
    b.C = restrict_active ? e : Pn; b.ldc = n;
    b.mirror = 1;  // X Pi X^dagger is Hermitian
    gemm(b, s, wk(), wcap());
    if (restrict_active) {
      kramers_even_kernel<<<blocks_for(n2), 256, 0, s>>>(Pn, e, n, nb);
      RR_LAUNCH_CHECK();
    }
    maxdiff_partial_kernel<2><<<RED_CTAS, 256, 0, s>>>(Pn, P, n2, red);
    RR_LAUNCH_CHECK();
    reduce_partials_kernel<2><<<1, 256, 0, s>>>(red, RED_CTAS, 1.0, scal + 1);
    RR_LAUNCH_CHECK();
    pt.mark(3, s);
    double hv[2];
    RR_CUDA(cudaMemcpyAsync(hv, scal, sizeof(hv), cudaMemcpyDeviceToHost, s));
    host_wait(h, s);
    pt.accumulate();
    const double energy = hv[0], dP = hv[1], dE = std::fabs(energy - prev);
    if (hist) hist[it - 1] = energy;
    res->electronic_energy = energy;
    const bool conv = it > 1 && (dP < so->density_tolerance || dE < so->energy_tolerance);
    prev = energy;
    if (conv) {
      if (mixed) {
        // last iteration in FP64: the FP64 energy of the newest density.  Unless the caller asked for
        // the Fock matrix or orbitals, only the energy is formed: J in FP64 and the FP64 half-transform
        // give 1/2 Re Tr[P (h + F)] = Re Tr[P h] + E_J - E_K / 2 without the exchange products.
        if (mixing_on) axpby(Pn, P, 1.0 - so->mixing, so->mixing, c2, s);
        have_proj = !mixing_on;
        std::swap(P, Pn);
        // (with linear mixing the density is not c_t^dagger c_t, so the full build gives its energy)
        const bool full_fock = res->fock_matrix || res->c_matrix || res->orbital_energies || mixing_on;
        pt.mark(0, s);
        double ev = 0.0;
        if (full_fock) {
          build(nullptr);
          pt.mark(1, s);
          energy_of_f();
          RR_CUDA(cudaMemcpyAsync(&ev, scal, sizeof(double), cudaMemcpyDeviceToHost, s));
        } else {
          RelBuild rb;
          rb.energy = scal + 24;
          build(&rb);
          pt.mark(1, s);
          // Re Tr[P h] = 1/2 sum_ij P_ij (h + h)_ji
          energy_partial_kernel<2><<<RED_CTAS, 256, 0, s>>>(P, hd, hd, n, red);
          RR_LAUNCH_CHECK();
          reduce_partials_kernel<0><<<1, 256, 0, s>>>(red, RED_CTAS, 0.5, scal + 26);
          RR_LAUNCH_CHECK();
          double e3[3];
          RR_CUDA(cudaMemcpyAsync(e3, scal + 24, sizeof(e3), cudaMemcpyDeviceToHost, s));
          host_wait(h, s);
          ev = e3[2] + e3[0] - 0.5 * e3[1];
        }
        ++n_fp64;
        host_wait(h, s);
        pt.accumulate_build();
        res->electronic_energy = ev;
        if (it < so->max_iterations) {
          ++it;
          if (hist) hist[it - 1] = ev;
        }
      }
      converged = true;
      break;
    }
    if (mixed && !reseeded && so->mixed_switch > 0.0 && it > 1 && dE < so->mixed_switch) reseed = reseeded = true;
    if (mixing_on) axpby(Pn, P, 1.0 - so->mixing, so->mixing, c2, s);
    have_proj = !mixing_on;
    std::swap(P, Pn);
  }
  if (it > so->max_iterations) it = so->max_iterations;
  scf_result_outputs(h, mixed && converged ? F : Fs, Xd, n, n_eff, true, res, host, s);
  check_status(h, s);
  copy_out(P_out, P, c2, host, s);
  host_wait(h, s);
  res->iterations = it;
  res->converged = converged ? 1 : 0;
  res->mixed_iterations = n_mixed;
  res->fp64_iterations = n_fp64;
  res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  pt.store(res);
}

}  // namespace rr
