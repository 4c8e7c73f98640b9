// Orbital-rotation optimisation of the functional stage on the GPU (reference: src/Utils/ADAM.cpp,
// the ADAM branch of the orbital optimisation, and the RotationProblem of
// src/Full_opt/FullOptimization.cpp:1330-1548) with a fixed-occupation hartree-exchange functional
// (two_rdm_h / two_rdm_x and the optional pair terms two_rdm_l1 / two_rdm_l2), for either MO tensor:
// the nonrelativistic spin-orbital RiNonRelSpinMoEri (RotationProblem<double, ...>) or the complex
// spinor RiMoEri of X2C / 4c (RotationProblem<complex<double>, ...>).
//
// Per ADAM step, all on the device:
//   g_I = 2 (F_qp - conj F_pq) over the pairs (p > q): for the spin-orbital kind the 2n spin
//         orbitals with twin pairs (the same spatial pair in the other spin) averaged; for the
//         complex kind the n spinors minus the pairs touching the first n_negative ones
//         (excludeNegative, C4_DHF)                        (OrbitalGradient.h, FullOptimization.cpp:1410)
//   step = Adam<T>::step(g)                                   (ADAM.cpp:33-51, exact IEEE operation order)
//   u = exp(-kappa), kappa_pq = step_I, kappa_qp = -conj step_I (ADAM.cpp:92-128); the spatial block
//         for the spin-orbital kind                        (SpinorRotation.cpp: eigen route there;
//         scaling and squaring of a Taylor series here, both equal to ~1e-15)
//   B^P <- u^dagger B^P u, h <- u^dagger h u, U_total <- U_total u   (RiNonRelSpinMoEri / RiMoEri ::rotated)
//   F = riHxFockGemm(h, B, occupations, two-RDMs)              (mo_hx_fock)
//   E = 1/2 sum_q [n_q Re h_qq + Re F_qq]                      (FullOptimization.cpp:1383)
// The run / restart / learning-rate logic of AdamOptimizer::run (ADAM.cpp:140-213) is host code.
//
// A learned preconditioner enters exactly where the reference's min-max stage rescales its pairs
// (FullOptimization.cpp:1362-1369): with per-pair scales s_I the optimiser sees g_I / sqrt(s_I) and
// the rotation uses step_I / sqrt(s_I) (ADAM runs in the variables sqrt(s) kappa).  Without scales it
// is plain ADAM.
#include <chrono>
#include <cmath>
#include <vector>

#include "gemm_f64.cuh"
#include "mo_store.cuh"

namespace rr {

namespace {

int blocks_for(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 1184))); }

__device__ __forceinline__ void pair_of_index(int64_t I, int64_t& p, int64_t& q) {
  // adamPairIndices order: (1,0), (2,0), (2,1), (3,0), ...: I = p (p - 1) / 2 + q
  p = static_cast<int64_t>((1.0 + sqrt(1.0 + 8.0 * static_cast<double>(I))) * 0.5);
  while (p * (p - 1) / 2 > I) --p;
  while ((p + 1) * p / 2 <= I) ++p;
  q = I - p * (p - 1) / 2;
}

// Adam<T>::step (ADAM.cpp:33-51) with the reference's operation order and no fused multiply-adds,
// so the device steps equal the host ones bit for bit.  PL = 2: complex entries (complex first
// moment, shared real second moment of |g|^2).
template <int PL>
__global__ void adam_step_kernel(double* m1, double* m2, double* mx, const double* g, double* out, int64_t n,
                                 double neg_lr, double b1, double omb1, double b2, double omb2, double c1, double c2,
                                 double eps) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double gr = g[i * PL], gi = PL == 2 ? g[i * PL + 1] : 0.0;
    const double ar = __dadd_rn(__dmul_rn(b1, m1[i * PL]), __dmul_rn(omb1, gr));
    m1[i * PL] = ar;
    double ai = 0.0;
    if (PL == 2) {
      ai = __dadd_rn(__dmul_rn(b1, m1[i * PL + 1]), __dmul_rn(omb1, gi));
      m1[i * PL + 1] = ai;
    }
    const double sq = PL == 2 ? __dadd_rn(__dmul_rn(gr, gr), __dmul_rn(gi, gi)) : __dmul_rn(gr, gr);
    const double v = __dadd_rn(__dmul_rn(b2, m2[i]), __dmul_rn(omb2, sq));
    m2[i] = v;
    const double vh = __ddiv_rn(v, c2);
    const double mv = mx[i] < vh ? vh : mx[i];
    mx[i] = mv;
    const double den = __dadd_rn(__dsqrt_rn(mv), eps);
    out[i * PL] = __ddiv_rn(__dmul_rn(neg_lr, __ddiv_rn(ar, c1)), den);
    if (PL == 2) out[i * PL + 1] = __ddiv_rn(__dmul_rn(neg_lr, __ddiv_rn(ai, c1)), den);
  }
}

// Pair gradient of the spin-orbital problem: g_I = 2 (F_qp - F_pq), averaged with the twin pair
// (spin partner x -> (x + n) mod 2n) when that is again a p > q pair; divided by sqrt(scale_I).
__global__ void pair_gradient_kernel(const double* F, int64_t n, int64_t npairs, const double* scale, double* g) {
  const int64_t d = 2 * n;
  for (int64_t I = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; I < npairs;
       I += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int64_t p, q;
    pair_of_index(I, p, q);
    double v = 2.0 * (F[q * d + p] - F[p * d + q]);
    const int64_t pp = (p + n) % d, qq = (q + n) % d;
    if (pp > qq) v = 0.5 * (v + 2.0 * (F[qq * d + pp] - F[pp * d + qq]));
    g[I] = scale ? v / sqrt(scale[I]) : v;
  }
}

// out[0] = max |g| (one CTA)
__global__ void absmax_kernel(const double* g, int64_t n, double* out) {
  __shared__ double red[32];
  double m = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, fabs(g[i]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    out[0] = m;
  }
}

// Spatial kappa (n x n) from the alpha-alpha pairs (p, q < n): kappa_pq = step_I / sqrt(scale_I),
// kappa_qp = -kappa_pq; out[0] = max_i sum_j |kappa_ij| (1-norm bound for the scaling).
__global__ void kappa_kernel(const double* step, const double* scale, int64_t n, double* kappa, double* norm) {
  __shared__ double red[32];
  double m = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    double r = 0.0;
    for (int64_t j = 0; j < n; ++j) {
      double v = 0.0;
      if (i != j) {
        const int64_t p = i > j ? i : j, q = i > j ? j : i;
        const int64_t I = p * (p - 1) / 2 + q;
        const double s = scale ? step[I] / sqrt(scale[I]) : step[I];
        v = i > j ? s : -s;
      }
      kappa[i * n + j] = v;
      r += fabs(v);
    }
    m = fmax(m, r);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    norm[0] = m;
  }
}

// Y = I + c X (n x n, real)
__global__ void eye_plus_kernel(double* Y, const double* X, double c, int64_t n) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < n * n;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x)
    Y[idx] = (idx / n == idx % n ? 1.0 : 0.0) + c * X[idx];
}

// H (2n x 2n) = blockdiag(h, h) from the spatial h (n x n)
__global__ void spin_block_kernel(const double* h, int64_t n, double* H) {
  const int64_t d = 2 * n;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < d * d;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t a = idx / d, b = idx % d;
    H[idx] = (a < n) == (b < n) ? h[(a % n) * n + (b % n)] : 0.0;
  }
}

// out[0] = 1/2 sum_q [n_q H_qq + F_qq] (one CTA)
__global__ void energy_trace_kernel(const double* H, const double* F, const double* occ, int64_t d, double* out) {
  __shared__ double red[32];
  double a = 0.0;
  for (int64_t q = threadIdx.x; q < d; q += blockDim.x) a += occ[q] * H[q * d + q] + F[q * d + q];
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += red[w];
    out[0] = 0.5 * t;
  }
}

// eri(a,b,c,d) = sum_P B(P, a%n c%n) B(P, b%n d%n), zero unless spin a == spin c and spin b == spin d
// (RiNonRelSpinMoEri::operator(), src/NON_REL/NonRelSpinRiMoEri.h:40); one warp, fixed order.
__device__ double eri_warp(const double* B, int64_t naux, int64_t n, int64_t a, int64_t b, int64_t c, int64_t d) {
  if ((a < n) != (c < n) || (b < n) != (d < n)) return 0.0;
  const int64_t ac = (a % n) * n + (c % n), bd = (b % n) * n + (d % n), nn = n * n;
  double s = 0.0;
  for (int64_t P = threadIdx.x & 31; P < naux; P += 32) s = fma(B[P * nn + ac], B[P * nn + bd], s);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

struct HessArgs {
  const double* H;   // d x d
  const double* F;   // d x d
  const double* occ;
  const double* h2;
  const double* x2;
  const double* J;   // J_ab = eri(a,b,a,b)
  const double* K;   // K_ab = eri(a,b,b,a) (= eri(a,a,b,b) for symmetric B^P)
  const double* M1;  // h2 (K - J)
  const double* B;   // spatial MO tensor (L terms)
  const int64_t* po;
  const double* l1;
  const double* l2;
  int64_t n, d, naux, npairs;
  double* out;
};

// Bare L1/L2 term of G_pq,rs (HartreeExchangeHessian.cpp:124-161), one warp.
__device__ double raw_l_warp(const HessArgs& a, int64_t p, int64_t q, int64_t r, int64_t s) {
  const int64_t* po = a.po;
  const int64_t d = a.d;
  double t = 0.0;
  if (q == po[s]) {
    double sum = 0.0;
    for (int64_t u = 0; u < d; ++u)
      sum += eri_warp(a.B, a.naux, a.n, u, po[u], p, r) * (a.l1[u * d + s] + a.l2[u * d + q]);
    t -= 2.0 * sum;
  }
  {
    const double c = a.l1[r * d + q] + a.l2[r * d + po[q]];
    t += 2.0 * eri_warp(a.B, a.naux, a.n, po[r], s, p, po[q]) * c;
    t -= 2.0 * eri_warp(a.B, a.naux, a.n, s, po[r], p, po[q]) * c;
  }
  {
    const double c = a.l1[p * d + s] + a.l2[p * d + po[s]];
    t += 2.0 * eri_warp(a.B, a.naux, a.n, po[p], q, r, po[s]) * c;
    t -= 2.0 * eri_warp(a.B, a.naux, a.n, po[p], q, po[s], r) * c;
  }
  if (p == po[r]) {
    double sum = 0.0;
    for (int64_t w = 0; w < d; ++w)
      sum += eri_warp(a.B, a.naux, a.n, s, q, w, po[w]) * (a.l1[r * d + w] + a.l2[r * d + po[w]]);
    t += 2.0 * sum;
  }
  return t;
}

// hartreeExchangeHessianElement(p,q,p,q) (HartreeExchangeHessian.cpp:221) for every pair p > q:
// the four bare H/X terms of the antisymmetrised diagonal reduce to J, K, F, h and
// M1 = two_rdm_h (K - J) entries (no sums left); the L1/L2 part evaluates its integrals directly.
// One warp per pair.
__global__ void hessian_diag_kernel(const HessArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  const int64_t d = a.d;
  for (int64_t I = warp; I < a.npairs; I += nw) {
    int64_t p, q;
    pair_of_index(I, p, q);
    auto H = [&](int64_t i, int64_t j) { return a.H[i * d + j]; };
    auto F = [&](int64_t i, int64_t j) { return a.F[i * d + j]; };
    auto h2 = [&](int64_t i, int64_t j) { return a.h2[i * d + j]; };
    auto x2 = [&](int64_t i, int64_t j) { return a.x2[i * d + j]; };
    auto J = [&](int64_t i, int64_t j) { return a.J[i * d + j]; };
    auto K = [&](int64_t i, int64_t j) { return a.K[i * d + j]; };
    auto M1 = [&](int64_t i, int64_t j) { return a.M1[i * d + j]; };
    const double np = a.occ[p], nq = a.occ[q];
    // raw(p,q,p,q): no delta terms; eri(q,q,p,p) twice
    const double r1 = K(q, p) * (x2(p, q) - h2(q, q) + x2(p, q) - x2(p, p)) +
                      K(q, p) * (h2(p, p) + x2(q, q) - x2(p, q) - x2(p, q));
    // raw(p,q,q,p)
    const double r2 = F(p, p) - H(p, p) * nq + M1(q, p) + F(q, q) - H(q, q) * np + M1(p, q) +
                      J(p, q) * (x2(q, q) - h2(p, q) + x2(p, p) - x2(q, p)) +
                      K(p, q) * (h2(q, p) + x2(q, p) - x2(p, p) - x2(q, q));
    // raw(q,p,p,q)
    const double r3 = F(q, q) - H(q, q) * np + M1(p, q) + F(p, p) - H(p, p) * nq + M1(q, p) +
                      J(q, p) * (x2(p, p) - h2(q, p) + x2(q, q) - x2(p, q)) +
                      K(q, p) * (h2(p, q) + x2(p, q) - x2(q, q) - x2(p, p));
    // raw(q,p,q,p): eri(p,p,q,q) twice
    const double r4 = K(p, q) * (x2(q, p) - h2(p, p) + x2(q, p) - x2(q, q)) +
                      K(p, q) * (h2(q, q) + x2(p, p) - x2(q, p) - x2(q, p));
    double v = r1 - r2 - r3 + r4;
    if (a.po) {
      v += raw_l_warp(a, p, q, p, q) - raw_l_warp(a, p, q, q, p) - raw_l_warp(a, q, p, p, q) +
           raw_l_warp(a, q, p, q, p);
    }
    if (lane == 0) a.out[I] = v;
  }
}

// Preconditioner features per pair I = (p, q), i = q, a = p:
// [F_ii, F_aa, n_i, n_a, J_ia, K_ia, J_ii, J_aa] (F: generalized Fock diagonal, the orbital-energy
// analogue of the functional stage), FP32.
__global__ void features_kernel(const double* F, const double* occ, const double* J, const double* K, int64_t d,
                                int64_t npairs, float* out) {
  for (int64_t I = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; I < npairs;
       I += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int64_t p, q;
    pair_of_index(I, p, q);
    float* o = out + I * 8;
    o[0] = static_cast<float>(F[q * d + q]);
    o[1] = static_cast<float>(F[p * d + p]);
    o[2] = static_cast<float>(occ[q]);
    o[3] = static_cast<float>(occ[p]);
    o[4] = static_cast<float>(J[q * d + p]);
    o[5] = static_cast<float>(K[q * d + p]);
    o[6] = static_cast<float>(J[q * d + q]);
    o[7] = static_cast<float>(J[p * d + p]);
  }
}

// ---- complex (RiMoEri) problem: explicit pair table pq[2I] = p, pq[2I+1] = q (p > q), interleaved
// complex matrices.

// g_I = 2 (F_qp - conj F_pq) (orbitalGradient, src/Hessian_opt/OrbitalGradient.h), divided by
// sqrt(scale_I) on both components.
__global__ void pair_gradient_c_kernel(const double* F, int64_t d, int64_t npairs, const int64_t* pq,
                                       const double* scale, double* g) {
  for (int64_t I = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; I < npairs;
       I += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t p = pq[2 * I], q = pq[2 * I + 1];
    double re = 2.0 * (F[2 * (q * d + p)] - F[2 * (p * d + q)]);
    double im = 2.0 * (F[2 * (q * d + p) + 1] + F[2 * (p * d + q) + 1]);
    if (scale) {
      const double r = sqrt(scale[I]);
      re /= r;
      im /= r;
    }
    g[2 * I] = re;
    g[2 * I + 1] = im;
  }
}

// out[0] = max |g_I| (complex modulus; one CTA)
__global__ void absmax_c_kernel(const double* g, int64_t n, double* out) {
  __shared__ double red[32];
  double m = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, hypot(g[2 * i], g[2 * i + 1]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    out[0] = m;
  }
}

// adamKappaMatrix (src/Utils/ADAM.cpp:106-128) over the pair table: kappa_pq = step_I / sqrt(scale_I),
// kappa_qp = -conj(kappa_pq); kappa zeroed beforehand.
__global__ void kappa_c_scatter_kernel(const double* step, const double* scale, const int64_t* pq, int64_t npairs,
                                       int64_t n, double* kappa) {
  for (int64_t I = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; I < npairs;
       I += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t p = pq[2 * I], q = pq[2 * I + 1];
    double re = step[2 * I], im = step[2 * I + 1];
    if (scale) {
      const double r = sqrt(scale[I]);
      re /= r;
      im /= r;
    }
    kappa[2 * (p * n + q)] = re;
    kappa[2 * (p * n + q) + 1] = im;
    kappa[2 * (q * n + p)] = -re;
    kappa[2 * (q * n + p) + 1] = im;
  }
}

// out[0] = max_i sum_j |kappa_ij| (complex modulus; one CTA)
__global__ void row_norm_c_kernel(const double* kappa, int64_t n, double* out) {
  __shared__ double red[32];
  double m = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    double r = 0.0;
    for (int64_t j = 0; j < n; ++j) r += hypot(kappa[2 * (i * n + j)], kappa[2 * (i * n + j) + 1]);
    m = fmax(m, r);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    out[0] = m;
  }
}

// Y = I + c X (n x n, interleaved complex, c real)
__global__ void eye_plus_c_kernel(double* Y, const double* X, double c, int64_t n) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < n * n;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    Y[2 * idx] = (idx / n == idx % n ? 1.0 : 0.0) + c * X[2 * idx];
    Y[2 * idx + 1] = c * X[2 * idx + 1];
  }
}

// out[0] = 1/2 sum_q [n_q Re H_qq + Re F_qq] (FullOptimization.cpp:1383; one CTA, interleaved complex)
__global__ void energy_trace_c_kernel(const double* H, const double* F, const double* occ, int64_t d, double* out) {
  __shared__ double red[32];
  double a = 0.0;
  for (int64_t q = threadIdx.x; q < d; q += blockDim.x) a += occ[q] * H[2 * (q * d + q)] + F[2 * (q * d + q)];
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += red[w];
    out[0] = 0.5 * t;
  }
}

// Preconditioner inputs of the complex problem (real parts of the complex F, J, K), FP32.
__global__ void features_c_kernel(const double* F, const double* occ, const double* J, const double* K, int64_t d,
                                  int64_t npairs, const int64_t* pq, float* out) {
  for (int64_t I = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; I < npairs;
       I += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t p = pq[2 * I], q = pq[2 * I + 1];
    float* o = out + I * 8;
    o[0] = static_cast<float>(F[2 * (q * d + q)]);
    o[1] = static_cast<float>(F[2 * (p * d + p)]);
    o[2] = static_cast<float>(occ[q]);
    o[3] = static_cast<float>(occ[p]);
    o[4] = static_cast<float>(J[2 * (q * d + p)]);
    o[5] = static_cast<float>(K[2 * (q * d + p)]);
    o[6] = static_cast<float>(J[2 * (q * d + q)]);
    o[7] = static_cast<float>(J[2 * (p * d + p)]);
  }
}

// Quadratic test problem E(x) = sum (a x^2/2 + b x) + c (sum x^2)^2 (one CTA each).
__global__ void quad_energy_kernel(const double* x, const double* a, const double* b, double c, int64_t n, double* out) {
  __shared__ double red[2][32];
  double e = 0.0, r = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    e += 0.5 * a[i] * x[i] * x[i] + b[i] * x[i];
    r += x[i] * x[i];
  }
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_xor_sync(0xffffffffu, e, o);
    r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = e; red[1][threadIdx.x >> 5] = r; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double te = 0.0, tr = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) { te += red[0][w]; tr += red[1][w]; }
    out[0] = te + c * tr * tr;
    out[1] = tr;
  }
}

__global__ void quad_gradient_kernel(const double* x, const double* a, const double* b, double c, const double* r2,
                                     int64_t n, double* g) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    g[i] = a[i] * x[i] + b[i] + 4.0 * c * r2[0] * x[i];
}

}  // namespace

// ------------------------------------------------------------------------------------ ADAM state

struct DeviceAdam {
  int64_t n = 0;
  int PL = 1;
  int t = 0;
  double lr = 0.01, b1 = 0.7, b2 = 0.9, eps = 1e-15;
  DevBuf<double> m1, m2, mx;
  void init(int64_t count, int pl, const rr_adam_options& o, double rate, cudaStream_t s) {
    n = count;
    PL = pl;
    b1 = o.beta1;
    b2 = o.beta2;
    eps = o.epsilon;
    lr = rate;
    m1.ensure(static_cast<size_t>(std::max<int64_t>(PL * n, 1)));
    m2.ensure(static_cast<size_t>(std::max<int64_t>(n, 1)));
    mx.ensure(static_cast<size_t>(std::max<int64_t>(n, 1)));
    clean(s);
  }
  void clean(cudaStream_t s) {
    t = 0;
    if (n) {
      RR_CUDA(cudaMemsetAsync(m1.p, 0, sizeof(double) * PL * n, s));
      RR_CUDA(cudaMemsetAsync(m2.p, 0, sizeof(double) * n, s));
      RR_CUDA(cudaMemsetAsync(mx.p, 0, sizeof(double) * n, s));
    }
  }
  void step(const double* g, double* out, cudaStream_t s) {
    ++t;
    const double c1 = 1.0 - std::pow(b1, t), c2 = 1.0 - std::pow(b2, t);
    if (!n) return;
    if (PL == 2)
      adam_step_kernel<2><<<blocks_for(n), 256, 0, s>>>(m1.p, m2.p, mx.p, g, out, n, -lr, b1, 1.0 - b1, b2, 1.0 - b2, c1,
                                                        c2, eps);
    else
      adam_step_kernel<1><<<blocks_for(n), 256, 0, s>>>(m1.p, m2.p, mx.p, g, out, n, -lr, b1, 1.0 - b1, b2, 1.0 - b2, c1,
                                                        c2, eps);
    RR_LAUNCH_CHECK();
  }
};

// What AdamOptimizer::run needs from a problem (AdamProblem, ADAM.h:153-180), device side.
struct OptProblem {
  virtual ~OptProblem() = default;
  virtual int64_t dim() const = 0;
  virtual int pl() const { return 1; }           // 2: complex parameters (interleaved)
  virtual double energy() = 0;                   // trial point
  virtual double gradient(double* g) = 0;        // g on the device; returns max |g|
  virtual void rotate(const double* step) = 0;   // step on the device
  virtual void save_best() = 0;
  virtual void restore_best() = 0;
  virtual cudaStream_t stream() const = 0;
};

// AdamOptimizer<double> (ADAM.cpp:133-213): the state that persists across runs.
struct OptState {
  rr_adam_options opt{};
  double lr = 0.01;
  int extra = 0;
  bool restart = false;
  DeviceAdam adam;
  DevBuf<double> g, step;
};

rr_adam_options default_adam_options() {
  rr_adam_options o{};
  o.learning_rate = 0.01;
  o.rate_factor = 0.2;
  o.beta1 = 0.7;
  o.beta2 = 0.9;
  o.epsilon = 1e-15;
  o.base_iterations = 10;
  o.iterations_increment = 20;
  o.max_iterations_limit = 200;
  o.gradient_tolerance = 1e-5;
  o.energy_tolerance = 1e-9;
  return o;
}

rr_adam_result adam_run(OptState& st, OptProblem& prob) {
  rr_adam_result res{};
  cudaStream_t s = prob.stream();
  st.restart = false;
  int max_calls = st.opt.base_iterations + st.extra;
  if (max_calls > st.opt.max_iterations_limit) max_calls = st.opt.base_iterations;
  const int64_t n = prob.dim();
  const int PL = prob.pl();
  st.g.ensure(static_cast<size_t>(std::max<int64_t>(PL * n, 1)));
  st.step.ensure(static_cast<size_t>(std::max<int64_t>(PL * n, 1)));
  st.adam.init(n, PL, st.opt, st.lr, s);
  res.learning_rate = st.lr;
  double e_old = prob.energy();
  double e_best = e_old;
  prob.save_best();
  double ediff = 0.0, maxg_best = 0.0, maxg = 0.0;
  res.energy_start = e_old;
  for (;;) {
    maxg = prob.gradient(st.g.p);
    if (maxg < st.opt.gradient_tolerance) {
      res.gradient_converged = 1;
      st.lr = st.opt.learning_rate;
      st.extra = 0;
      break;
    }
    st.adam.step(st.g.p, st.step.p, s);
    prob.rotate(st.step.p);
    const double e = prob.energy();
    if (e < e_best) {
      res.improved = 1;
      e_best = e;
      maxg_best = maxg;
      prob.save_best();
    }
    ediff = e - e_old;
    if (st.adam.t > 1 && std::fabs(ediff) < st.opt.energy_tolerance) {
      res.energy_converged = 1;
      break;
    }
    e_old = e;
    if (st.adam.t == max_calls) break;
  }
  res.iterations = st.adam.t;
  res.energy_best = e_best;
  res.energy_difference = ediff;
  res.max_gradient = res.improved ? maxg_best : maxg;
  if (!res.improved && std::fabs(ediff) > st.opt.energy_tolerance) {
    st.restart = true;
    st.lr *= st.opt.rate_factor;
    st.extra += st.opt.iterations_increment;
  }
  res.restart_requested = st.restart ? 1 : 0;
  prob.restore_best();
  return res;
}

// U = exp(-kappa) for an anti-symmetric (real) or anti-Hermitian (complex, interleaved) n x n kappa
// on the device, by scaling and squaring of the Taylor series in Horner form: after scaling
// ||A|| <= 1/2 (norm = a 1-norm bound of kappa) and the degree is the smallest m with
// ||A||^(m+1) / (m+1)! < 2^-60.  Ta, Tb: n x n scratch of the same element kind.
// (src/Hessian_opt/SpinorRotation.cpp:17 forms the same matrix through the eigenvectors of i kappa.)
void expm_neg(const double* kap, double norm, int64_t n, double* U, double* Ta, double* Tb, cudaStream_t s,
              bool cplx) {
  int sq = 0;
  double a = norm;
  while (a > 0.5) { a *= 0.5; ++sq; }
  int m = 1;
  double term = a;
  while (m < 30) {
    term *= a / (m + 1);
    if (term < 8.7e-19) break;
    ++m;
  }
  const double scale = -std::ldexp(1.0, -sq);  // A = -kappa / 2^sq
  auto eye_plus = [&](double* Y, const double* X, double c) {
    if (cplx) eye_plus_c_kernel<<<blocks_for(n * n), 256, 0, s>>>(Y, X, c, n);
    else eye_plus_kernel<<<blocks_for(n * n), 256, 0, s>>>(Y, X, c, n);
    RR_LAUNCH_CHECK();
  };
  GemmDesc g;
  g.cplx = cplx;
  g.M = n; g.N = n; g.K = n; g.A = kap; g.lda = n; g.ldb = n; g.ldc = n;
  eye_plus(Ta, kap, scale / m);  // T = I + A/m
  for (int k = m - 1; k >= 1; --k) {  // T = I + (A T) / k
    g.B = Ta; g.C = Tb; g.alpha = scale / k; g.beta = 0.0;
    gemm(g, s);
    eye_plus(Ta, Tb, 1.0);
  }
  for (int i = 0; i < sq; ++i) {
    GemmDesc q;
    q.cplx = cplx;
    q.M = n; q.N = n; q.K = n; q.A = Ta; q.lda = n; q.B = Ta; q.ldb = n; q.C = Tb; q.ldc = n;
    gemm(q, s);
    std::swap(Ta, Tb);
  }
  RR_CUDA(cudaMemcpyAsync(U, Ta, sizeof(double) * (cplx ? 2 : 1) * n * n, cudaMemcpyDeviceToDevice, s));
}

}  // namespace rr
// ------------------------------------------------------------------ rotation problem (NON_REL RI)

struct rr_orbopt_store : rr::OptProblem {
  rr::Context ctx;
  // cplx 0: RiNonRelSpinMoEri (n spatial orbitals, d = 2n spin orbitals, pairs adamPairIndices(2n) by
  // formula, spin-restricted rotations of the spatial block); cplx 1: RiMoEri (d = n spinors, the
  // pair table pqd = adamPairIndices(n) without the pairs that touch the first n_negative spinors,
  // unitary rotations).
  int cplx = 0, PL = 1;
  int64_t n = 0, d = 0, naux = 0, npairs = 0, n_negative = 0;
  rr_mo_store mo;  // trial tensor (mo.B) and the MO kernels' scratch
  rr::DevBuf<double> Bbest, Bwork, mats;
  rr::DevBuf<int64_t> pqd;
  double *h_t = nullptr, *h_b = nullptr, *u_t = nullptr, *u_b = nullptr, *H = nullptr, *F = nullptr;
  double *occ = nullptr, *h2 = nullptr, *x2 = nullptr, *l1 = nullptr, *l2 = nullptr, *scal = nullptr;
  double *kap = nullptr, *U = nullptr, *Ta = nullptr, *Tb = nullptr, *scales = nullptr, *J = nullptr, *K = nullptr;
  double *M1 = nullptr;
  int64_t* po = nullptr;
  bool have_l = false, have_scales = false, fock_valid = false;
  double energy_cache = 0.0;
  rr::OptState state;

  int64_t dim() const override { return npairs; }
  int pl() const override { return PL; }
  cudaStream_t stream() const override { return ctx.main; }

  // excludeNegative(adamPairIndices(n), n_negative) (FullOptimization.cpp:83-92) into pqd.
  void set_pairs(int64_t nneg) {
    std::vector<int64_t> t;
    t.reserve(static_cast<size_t>(n * (n - 1)));
    for (int64_t p = 0; p < n; ++p)
      for (int64_t q = 0; q < p; ++q)
        if (p >= nneg && q >= nneg) {
          t.push_back(p);
          t.push_back(q);
        }
    n_negative = nneg;
    npairs = static_cast<int64_t>(t.size() / 2);
    pqd.ensure(std::max<size_t>(t.size(), 2));
    if (!t.empty())
      RR_CUDA(cudaMemcpyAsync(pqd.p, t.data(), sizeof(int64_t) * t.size(), cudaMemcpyHostToDevice, ctx.main));
    RR_CUDA(cudaStreamSynchronize(ctx.main));
  }

  // F and E at the trial orbitals (cached until the next rotation).
  void build_fock() {
    if (fock_valid) return;
    cudaStream_t s = ctx.main;
    if (cplx) {
      rr::mo_hx_fock(&mo, h_t, occ, h2, x2, have_l ? po : nullptr, l1, l2, F, false, s);
      rr::energy_trace_c_kernel<<<1, 256, 0, s>>>(h_t, F, occ, d, scal);
    } else {
      rr::spin_block_kernel<<<rr::blocks_for(d * d), 256, 0, s>>>(h_t, n, H);
      RR_LAUNCH_CHECK();
      rr::mo_hx_fock(&mo, H, occ, h2, x2, have_l ? po : nullptr, l1, l2, F, false, s);
      rr::energy_trace_kernel<<<1, 256, 0, s>>>(H, F, occ, d, scal);
    }
    RR_LAUNCH_CHECK();
    double e;
    RR_CUDA(cudaMemcpyAsync(&e, scal, sizeof(double), cudaMemcpyDeviceToHost, s));
    RR_CUDA(cudaStreamSynchronize(s));
    energy_cache = e;
    fock_valid = true;
  }
  double energy() override {
    build_fock();
    return energy_cache;
  }
  double gradient(double* g) override {
    build_fock();
    cudaStream_t s = ctx.main;
    const double* sc = have_scales ? scales : nullptr;
    if (cplx) {
      if (npairs) {
        rr::pair_gradient_c_kernel<<<rr::blocks_for(npairs), 256, 0, s>>>(F, d, npairs, pqd.p, sc, g);
        RR_LAUNCH_CHECK();
      }
      rr::absmax_c_kernel<<<1, 512, 0, s>>>(g, npairs, scal + 1);
    } else {
      rr::pair_gradient_kernel<<<rr::blocks_for(npairs), 256, 0, s>>>(F, n, npairs, sc, g);
      RR_LAUNCH_CHECK();
      rr::absmax_kernel<<<1, 512, 0, s>>>(g, npairs, scal + 1);
    }
    RR_LAUNCH_CHECK();
    double m;
    RR_CUDA(cudaMemcpyAsync(&m, scal + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
    RR_CUDA(cudaStreamSynchronize(s));
    return m;
  }
  void rotate(const double* step) override {
    cudaStream_t s = ctx.main;
    const double* sc = have_scales ? scales : nullptr;
    if (cplx) {
      RR_CUDA(cudaMemsetAsync(kap, 0, sizeof(double) * 2 * n * n, s));
      if (npairs) {
        rr::kappa_c_scatter_kernel<<<rr::blocks_for(npairs), 256, 0, s>>>(step, sc, pqd.p, npairs, n, kap);
        RR_LAUNCH_CHECK();
      }
      rr::row_norm_c_kernel<<<1, 256, 0, s>>>(kap, n, scal + 2);
    } else {
      rr::kappa_kernel<<<1, 256, 0, s>>>(step, sc, n, kap, scal + 2);
    }
    RR_LAUNCH_CHECK();
    double norm;
    RR_CUDA(cudaMemcpyAsync(&norm, scal + 2, sizeof(double), cudaMemcpyDeviceToHost, s));
    RR_CUDA(cudaStreamSynchronize(s));
    rr::expm_neg(kap, norm, n, U, Ta, Tb, s, cplx != 0);
    const int64_t nn = n * n;
    // real: u^T (.) u; complex: U^dagger (.) U (RiNonRelSpinMoEri::rotated / RiMoEri::rotated)
    rr::GemmDesc a;  // W^P = u^dagger B^P
    a.cplx = cplx; a.conjA = cplx;
    a.M = n; a.N = n; a.K = n; a.A = U; a.lda = n; a.opA = rr::Op::T;
    a.B = mo.B.p; a.ldb = n; a.strideB = nn; a.C = Bwork.p; a.ldc = n; a.strideC = nn; a.batch = naux;
    rr::gemm(a, s);
    rr::GemmDesc b;  // B^P = W^P u
    b.cplx = cplx;
    b.M = n; b.N = n; b.K = n; b.A = Bwork.p; b.lda = n; b.strideA = nn; b.B = U; b.ldb = n;
    b.C = mo.B.p; b.ldc = n; b.strideC = nn; b.batch = naux;
    rr::gemm(b, s);
    rr::GemmDesc c;  // h = u^dagger h u
    c.cplx = cplx; c.conjA = cplx;
    c.M = n; c.N = n; c.K = n; c.A = U; c.lda = n; c.opA = rr::Op::T; c.B = h_t; c.ldb = n; c.C = Ta; c.ldc = n;
    rr::gemm(c, s);
    c.opA = rr::Op::N; c.conjA = 0; c.A = Ta; c.B = U; c.C = h_t;
    rr::gemm(c, s);
    c.A = u_t; c.B = U; c.C = Ta;  // U_total <- U_total u
    rr::gemm(c, s);
    RR_CUDA(cudaMemcpyAsync(u_t, Ta, sizeof(double) * PL * nn, cudaMemcpyDeviceToDevice, s));
    fock_valid = false;
  }
  void save_best() override {
    cudaStream_t s = ctx.main;
    RR_CUDA(cudaMemcpyAsync(Bbest.p, mo.B.p, sizeof(double) * PL * naux * n * n, cudaMemcpyDeviceToDevice, s));
    RR_CUDA(cudaMemcpyAsync(h_b, h_t, sizeof(double) * PL * n * n, cudaMemcpyDeviceToDevice, s));
    RR_CUDA(cudaMemcpyAsync(u_b, u_t, sizeof(double) * PL * n * n, cudaMemcpyDeviceToDevice, s));
  }
  void restore_best() override {
    cudaStream_t s = ctx.main;
    RR_CUDA(cudaMemcpyAsync(mo.B.p, Bbest.p, sizeof(double) * PL * naux * n * n, cudaMemcpyDeviceToDevice, s));
    RR_CUDA(cudaMemcpyAsync(h_t, h_b, sizeof(double) * PL * n * n, cudaMemcpyDeviceToDevice, s));
    RR_CUDA(cudaMemcpyAsync(u_t, u_b, sizeof(double) * PL * n * n, cudaMemcpyDeviceToDevice, s));
    fock_valid = false;
  }
  // J, K (2n x 2n, spin rule) and M1 = two_rdm_h (K - J) at the current orbitals (F built too; real kind).
  void jk_m1() {
    cudaStream_t s = ctx.main;
    build_fock();
    rr::mo_jkl(&mo, nullptr, J, K, nullptr, false, s);
    RR_CUDA(cudaMemcpyAsync(M1, K, sizeof(double) * d * d, cudaMemcpyDeviceToDevice, s));
    rr::axpby(M1, J, -1.0, 1.0, d * d, s);  // K - J
    rr::GemmDesc g;
    g.M = d; g.N = d; g.K = d; g.A = h2; g.lda = d; g.B = M1; g.ldb = d; g.C = Ta; g.ldc = d;
    rr::gemm(g, s);
    RR_CUDA(cudaMemcpyAsync(M1, Ta, sizeof(double) * d * d, cudaMemcpyDeviceToDevice, s));
  }
};

namespace {

// Quadratic test problem for the run / restart logic (same as the oracle bridge's).
struct QuadProblem : rr::OptProblem {
  cudaStream_t s = nullptr;
  int64_t n = 0;
  double c = 0.0;
  rr::DevBuf<double> buf;
  double *x = nullptr, *xb = nullptr, *a = nullptr, *b = nullptr, *scal = nullptr;
  int64_t dim() const override { return n; }
  cudaStream_t stream() const override { return s; }
  double energy() override {
    rr::quad_energy_kernel<<<1, 256, 0, s>>>(x, a, b, c, n, scal);
    RR_LAUNCH_CHECK();
    double e;
    RR_CUDA(cudaMemcpyAsync(&e, scal, sizeof(double), cudaMemcpyDeviceToHost, s));
    RR_CUDA(cudaStreamSynchronize(s));
    return e;
  }
  double gradient(double* g) override {
    rr::quad_energy_kernel<<<1, 256, 0, s>>>(x, a, b, c, n, scal);
    RR_LAUNCH_CHECK();
    rr::quad_gradient_kernel<<<rr::blocks_for(n), 256, 0, s>>>(x, a, b, c, scal + 1, n, g);
    RR_LAUNCH_CHECK();
    rr::absmax_kernel<<<1, 256, 0, s>>>(g, n, scal + 2);
    RR_LAUNCH_CHECK();
    double m;
    RR_CUDA(cudaMemcpyAsync(&m, scal + 2, sizeof(double), cudaMemcpyDeviceToHost, s));
    RR_CUDA(cudaStreamSynchronize(s));
    return m;
  }
  void rotate(const double* step) override { rr::axpby(x, step, 1.0, 1.0, n, s); }
  void save_best() override { RR_CUDA(cudaMemcpyAsync(xb, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s)); }
  void restore_best() override { RR_CUDA(cudaMemcpyAsync(x, xb, sizeof(double) * n, cudaMemcpyDeviceToDevice, s)); }
};

template <typename Fn>
int guarded(Fn&& f) {
  try {
    rr::set_last_error("");
    f();
    return RR_OK;
  } catch (const rr::Error& e) {
    rr::set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    rr::set_last_error("host allocation failed");
    return RR_ERR_NOMEM;
  } catch (const std::exception& e) {
    rr::set_last_error(e.what());
    return RR_ERR_CUDA;
  }
}

rr_orbopt_store* checked_opt(rr_orbopt_handle h) {
  if (!h) throw rr::Error(RR_ERR_ARG, "null orbital-optimisation handle");
  RR_CUDA(cudaSetDevice(h->ctx.device));
  return h;
}

}  // namespace

// ------------------------------------------------------------------------------------- C ABI

extern "C" {

int rr_adam_default_options(rr_adam_options* out) {
  return guarded([&] {
    RR_REQUIRE(out, RR_ERR_ARG, "rr_adam_default_options: null output");
    *out = rr::default_adam_options();
  });
}

int rr_orbopt_create(rr_mo_handle m, const double* h, const double* occupations, const double* two_rdm_h,
                     const double* two_rdm_x, const int64_t* pair_of, const double* two_rdm_l1,
                     const double* two_rdm_l2, const rr_adam_options* options, rr_orbopt_handle* out) {
  return guarded([&] {
    RR_REQUIRE(m && out && h && occupations && two_rdm_h && two_rdm_x, RR_ERR_ARG, "rr_orbopt_create: null argument");
    RR_REQUIRE(!pair_of || (two_rdm_l1 && two_rdm_l2), RR_ERR_ARG,
               "rr_orbopt_create: pair_of needs two_rdm_l1 and two_rdm_l2");
    RR_CUDA(cudaSetDevice(m->ctx.device));
    *out = nullptr;
    const int cplx = m->cplx ? 1 : 0, PL = cplx ? 2 : 1;
    const int64_t n = m->n, d = cplx ? n : 2 * n, nn = n * n, dd = d * d;
    if (pair_of)
      for (int64_t i = 0; i < d; ++i)
        RR_REQUIRE(pair_of[i] >= 0 && pair_of[i] < d, RR_ERR_ARG, "rr_orbopt_create: pair_of out of range");
    auto* o = new rr_orbopt_store();
    try {
      o->ctx.init(nullptr);
      o->cplx = cplx;
      o->PL = PL;
      o->n = n;
      o->d = d;
      o->naux = m->naux;
      o->state.opt = options ? *options : rr::default_adam_options();
      o->state.lr = o->state.opt.learning_rate;
      cudaStream_t s = o->ctx.main;
      if (cplx) o->set_pairs(0);
      else o->npairs = d * (d - 1) / 2;
      o->mo.cplx = cplx;
      o->mo.naux = o->naux;
      o->mo.n = n;
      const size_t bsz = static_cast<size_t>(std::max<int64_t>(PL * o->naux * nn, 1));
      o->mo.B.alloc(bsz);
      o->Bbest.alloc(bsz);
      o->Bwork.alloc(bsz);
      RR_CUDA(cudaMemcpyAsync(o->mo.B.p, m->B.p, sizeof(double) * PL * o->naux * nn, cudaMemcpyDeviceToDevice, s));
      const int64_t mat = PL * nn, big = std::max(PL * nn, dd);
      rr::Arena ar(&o->mats);
      ar.request(&o->h_t, mat);
      ar.request(&o->h_b, mat);
      ar.request(&o->u_t, mat);
      ar.request(&o->u_b, mat);
      ar.request(&o->kap, mat);
      ar.request(&o->U, mat);
      ar.request(&o->Ta, big);
      ar.request(&o->Tb, big);
      ar.request(&o->H, dd);
      ar.request(&o->F, PL * dd);
      ar.request(&o->J, PL * dd);
      ar.request(&o->K, PL * dd);
      ar.request(&o->M1, dd);
      ar.request(&o->occ, d);
      ar.request(&o->h2, dd);
      ar.request(&o->x2, dd);
      ar.request(&o->l1, dd);
      ar.request(&o->l2, dd);
      ar.request(&o->scales, std::max<int64_t>(o->npairs, d * (d - 1) / 2));
      double* pob;
      ar.request(&pob, d);
      ar.request(&o->scal, 64);
      ar.commit();
      o->po = reinterpret_cast<int64_t*>(pob);
      rr::copy_in(o->h_t, h, mat, true, s);
      std::vector<double> eye(static_cast<size_t>(mat), 0.0);
      for (int64_t i = 0; i < n; ++i) eye[static_cast<size_t>(PL * (i * n + i))] = 1.0;
      rr::copy_in(o->u_t, eye.data(), mat, true, s);
      rr::copy_in(o->occ, occupations, d, true, s);
      rr::copy_in(o->h2, two_rdm_h, dd, true, s);
      rr::copy_in(o->x2, two_rdm_x, dd, true, s);
      o->have_l = pair_of != nullptr;
      if (o->have_l) {
        rr::copy_in(o->l1, two_rdm_l1, dd, true, s);
        rr::copy_in(o->l2, two_rdm_l2, dd, true, s);
        RR_CUDA(cudaMemcpyAsync(o->po, pair_of, sizeof(int64_t) * d, cudaMemcpyHostToDevice, s));
      }
      RR_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
      o->ctx.destroy();
      delete o;
      throw;
    }
    *out = o;
  });
}

int rr_orbopt_exclude_negative(rr_orbopt_handle h, int64_t n_negative) {
  return guarded([&] {
    auto* o = checked_opt(h);
    RR_REQUIRE(o->cplx, RR_ERR_UNSUPPORTED,
               "rr_orbopt_exclude_negative: the negative-energy branch exists for the complex (4-component) tensor only");
    RR_REQUIRE(n_negative >= 0 && n_negative <= o->n, RR_ERR_ARG, "rr_orbopt_exclude_negative: n_negative out of range");
    o->set_pairs(n_negative);
    o->have_scales = false;
  });
}

int rr_orbopt_set_functional(rr_orbopt_handle h, const double* occupations, const double* two_rdm_h,
                             const double* two_rdm_x, const int64_t* pair_of, const double* two_rdm_l1,
                             const double* two_rdm_l2) {
  return guarded([&] {
    auto* o = checked_opt(h);
    RR_REQUIRE(occupations && two_rdm_h && two_rdm_x, RR_ERR_ARG, "rr_orbopt_set_functional: null argument");
    RR_REQUIRE(!pair_of || (two_rdm_l1 && two_rdm_l2), RR_ERR_ARG,
               "rr_orbopt_set_functional: pair_of needs two_rdm_l1 and two_rdm_l2");
    const int64_t d = o->d, dd = d * d;
    if (pair_of)
      for (int64_t i = 0; i < d; ++i)
        RR_REQUIRE(pair_of[i] >= 0 && pair_of[i] < d, RR_ERR_ARG, "rr_orbopt_set_functional: pair_of out of range");
    cudaStream_t s = o->ctx.main;
    rr::copy_in(o->occ, occupations, d, true, s);
    rr::copy_in(o->h2, two_rdm_h, dd, true, s);
    rr::copy_in(o->x2, two_rdm_x, dd, true, s);
    o->have_l = pair_of != nullptr;
    if (o->have_l) {
      rr::copy_in(o->l1, two_rdm_l1, dd, true, s);
      rr::copy_in(o->l2, two_rdm_l2, dd, true, s);
      RR_CUDA(cudaMemcpyAsync(o->po, pair_of, sizeof(int64_t) * d, cudaMemcpyHostToDevice, s));
    }
    RR_CUDA(cudaStreamSynchronize(s));
    o->fock_valid = false;
  });
}

int rr_orbopt_jk(rr_orbopt_handle h, double* J, double* K) {
  return guarded([&] {
    auto* o = checked_opt(h);
    RR_REQUIRE(J && K, RR_ERR_ARG, "rr_orbopt_jk: null output");
    rr::mo_jkl(&o->mo, nullptr, J, K, nullptr, true, o->ctx.main);
    RR_CUDA(cudaStreamSynchronize(o->ctx.main));
  });
}

int rr_orbopt_destroy(rr_orbopt_handle h) {
  return guarded([&] {
    if (!h) return;
    cudaSetDevice(h->ctx.device);
    h->ctx.destroy();
    delete h;
  });
}

int rr_orbopt_info(rr_orbopt_handle h, int64_t* n_pairs, int64_t* n_spatial, int64_t* naux) {
  return guarded([&] {
    auto* o = checked_opt(h);
    if (n_pairs) *n_pairs = o->npairs;
    if (n_spatial) *n_spatial = o->n;
    if (naux) *naux = o->naux;
  });
}

int rr_orbopt_set_scales(rr_orbopt_handle h, const double* scales) {
  return guarded([&] {
    auto* o = checked_opt(h);
    if (!scales) {
      o->have_scales = false;
      return;
    }
    for (int64_t i = 0; i < o->npairs; ++i)
      RR_REQUIRE(scales[i] > 0.0 && std::isfinite(scales[i]), RR_ERR_ARG,
                 "rr_orbopt_set_scales: scales must be positive and finite");
    rr::copy_in(o->scales, scales, o->npairs, true, o->ctx.main);
    RR_CUDA(cudaStreamSynchronize(o->ctx.main));
    o->have_scales = true;
  });
}

int rr_orbopt_run(rr_orbopt_handle h, rr_adam_result* result) {
  return guarded([&] {
    auto* o = checked_opt(h);
    RR_REQUIRE(result, RR_ERR_ARG, "rr_orbopt_run: null result");
    *result = rr::adam_run(o->state, *o);
    RR_CUDA(cudaStreamSynchronize(o->ctx.main));
  });
}

int rr_orbopt_energy(rr_orbopt_handle h, double* energy) {
  return guarded([&] {
    auto* o = checked_opt(h);
    RR_REQUIRE(energy, RR_ERR_ARG, "rr_orbopt_energy: null output");
    *energy = o->energy();
  });
}

int rr_orbopt_gradient(rr_orbopt_handle h, double* g) {
  return guarded([&] {
    auto* o = checked_opt(h);
    RR_REQUIRE(g, RR_ERR_ARG, "rr_orbopt_gradient: null output");
    rr::DevBuf<double> gd(static_cast<size_t>(std::max<int64_t>(o->PL * o->npairs, 1)));
    o->gradient(gd.p);
    rr::copy_out(g, gd.p, o->PL * o->npairs, true, o->ctx.main);
    RR_CUDA(cudaStreamSynchronize(o->ctx.main));
  });
}

int rr_orbopt_hessian_diagonal(rr_orbopt_handle h, double* out) {
  return guarded([&] {
    auto* o = checked_opt(h);
    RR_REQUIRE(out, RR_ERR_ARG, "rr_orbopt_hessian_diagonal: null output");
    cudaStream_t s = o->ctx.main;
    if (o->cplx) {
      // hartreeExchangeJointHessianDiagonal over the pair table: 2 n_pairs entries
      o->build_fock();
      rr::DevBuf<double> od(static_cast<size_t>(std::max<int64_t>(2 * o->npairs, 1)));
      rr::mo_hx_joint_hessian_diagonal(&o->mo, o->h_t, o->occ, o->h2, o->x2, o->F, o->npairs, o->pqd.p,
                                       o->have_l ? o->po : nullptr, o->l1, o->l2, od.p, false, s);
      rr::copy_out(out, od.p, 2 * o->npairs, true, s);
      RR_CUDA(cudaStreamSynchronize(s));
      return;
    }
    o->jk_m1();
    rr::spin_block_kernel<<<rr::blocks_for(o->d * o->d), 256, 0, s>>>(o->h_t, o->n, o->H);
    RR_LAUNCH_CHECK();
    rr::DevBuf<double> od(static_cast<size_t>(std::max<int64_t>(o->npairs, 1)));
    rr::HessArgs a{};
    a.H = o->H; a.F = o->F; a.occ = o->occ; a.h2 = o->h2; a.x2 = o->x2; a.J = o->J; a.K = o->K; a.M1 = o->M1;
    a.B = o->mo.B.p; a.po = o->have_l ? o->po : nullptr; a.l1 = o->l1; a.l2 = o->l2;
    a.n = o->n; a.d = o->d; a.naux = o->naux; a.npairs = o->npairs; a.out = od.p;
    const int64_t blocks = std::min<int64_t>(4096, (o->npairs + 7) / 8);
    rr::hessian_diag_kernel<<<static_cast<int>(std::max<int64_t>(blocks, 1)), 256, 0, s>>>(a);
    RR_LAUNCH_CHECK();
    rr::copy_out(out, od.p, o->npairs, true, s);
    RR_CUDA(cudaStreamSynchronize(s));
  });
}

int rr_orbopt_features(rr_orbopt_handle h, float* out) {
  return guarded([&] {
    auto* o = checked_opt(h);
    RR_REQUIRE(out, RR_ERR_ARG, "rr_orbopt_features: null output");
    cudaStream_t s = o->ctx.main;
    o->build_fock();
    rr::mo_jkl(&o->mo, nullptr, o->J, o->K, nullptr, false, s);
    rr::DevBuf<float> fd(static_cast<size_t>(std::max<int64_t>(8 * o->npairs, 1)));
    if (o->npairs) {
      if (o->cplx)
        rr::features_c_kernel<<<rr::blocks_for(o->npairs), 256, 0, s>>>(o->F, o->occ, o->J, o->K, o->d, o->npairs,
                                                                         o->pqd.p, fd.p);
      else
        rr::features_kernel<<<rr::blocks_for(o->npairs), 256, 0, s>>>(o->F, o->occ, o->J, o->K, o->d, o->npairs, fd.p);
      RR_LAUNCH_CHECK();
    }
    RR_CUDA(cudaMemcpyAsync(out, fd.p, sizeof(float) * 8 * o->npairs, cudaMemcpyDeviceToHost, s));
    RR_CUDA(cudaStreamSynchronize(s));
  });
}

int rr_orbopt_state(rr_orbopt_handle h, double* rotation, double* h_out, double* Bmo_out) {
  return guarded([&] {
    auto* o = checked_opt(h);
    cudaStream_t s = o->ctx.main;
    if (rotation) rr::copy_out(rotation, o->u_t, o->PL * o->n * o->n, true, s);
    if (h_out) rr::copy_out(h_out, o->h_t, o->PL * o->n * o->n, true, s);
    if (Bmo_out) rr::copy_out(Bmo_out, o->mo.B.p, o->PL * o->naux * o->n * o->n, true, s);
    RR_CUDA(cudaStreamSynchronize(s));
  });
}

// ---- test hooks (include/rr_ri_testing.h) ----

int rr_test_adam_steps(int64_t n, int32_t cplx, int64_t nsteps, double lr, double b1, double b2, double eps,
                       const double* grads, double* steps) {
  return guarded([&] {
    const int PL = cplx ? 2 : 1;
    cudaStream_t s = nullptr;
    rr_adam_options o = rr::default_adam_options();
    o.beta1 = b1;
    o.beta2 = b2;
    o.epsilon = eps;
    rr::DeviceAdam adam;
    adam.init(n, PL, o, lr, s);
    rr::DevBuf<double> g(static_cast<size_t>(std::max<int64_t>(PL * n, 1))), st(g.n);
    for (int64_t t = 0; t < nsteps; ++t) {
      RR_CUDA(cudaMemcpy(g.p, grads + t * PL * n, sizeof(double) * PL * n, cudaMemcpyHostToDevice));
      adam.step(g.p, st.p, s);
      RR_CUDA(cudaMemcpy(steps + t * PL * n, st.p, sizeof(double) * PL * n, cudaMemcpyDeviceToHost));
    }
  });
}

int rr_test_rotation_matrix(int64_t n, const double* kappa, double* U) {
  return guarded([&] {
    double norm = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      double r = 0.0;
      for (int64_t j = 0; j < n; ++j) r += std::fabs(kappa[i * n + j]);
      norm = std::max(norm, r);
    }
    rr::DevBuf<double> k(static_cast<size_t>(std::max<int64_t>(n * n, 1))), u(k.n), a(k.n), b(k.n);
    RR_CUDA(cudaMemcpy(k.p, kappa, sizeof(double) * n * n, cudaMemcpyHostToDevice));
    rr::expm_neg(k.p, norm, n, u.p, a.p, b.p, nullptr, false);
    RR_CUDA(cudaMemcpy(U, u.p, sizeof(double) * n * n, cudaMemcpyDeviceToHost));
  });
}

int rr_test_rotation_matrix_complex(int64_t n, const double* kappa, double* U) {
  return guarded([&] {
    double norm = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      double r = 0.0;
      for (int64_t j = 0; j < n; ++j) r += std::hypot(kappa[2 * (i * n + j)], kappa[2 * (i * n + j) + 1]);
      norm = std::max(norm, r);
    }
    const size_t cnt = static_cast<size_t>(std::max<int64_t>(2 * n * n, 2));
    rr::DevBuf<double> k(cnt), u(cnt), a(cnt), b(cnt);
    RR_CUDA(cudaMemcpy(k.p, kappa, sizeof(double) * 2 * n * n, cudaMemcpyHostToDevice));
    rr::expm_neg(k.p, norm, n, u.p, a.p, b.p, nullptr, true);
    RR_CUDA(cudaMemcpy(U, u.p, sizeof(double) * 2 * n * n, cudaMemcpyDeviceToHost));
  });
}

int rr_test_adam_run_quadratic(int64_t n, const double* a, const double* b, double c, const double* x0, int32_t runs,
                               double* energy_best, int32_t* iterations, int32_t* restart, double* rate,
                               double* x_out) {
  return guarded([&] {
    QuadProblem q;
    q.n = n;
    q.c = c;
    q.buf.alloc(static_cast<size_t>(4 * std::max<int64_t>(n, 1) + 8));
    q.x = q.buf.p;
    q.xb = q.x + n;
    q.a = q.xb + n;
    q.b = q.a + n;
    q.scal = q.b + n;
    RR_CUDA(cudaMemcpy(q.x, x0, sizeof(double) * n, cudaMemcpyHostToDevice));
    RR_CUDA(cudaMemcpy(q.a, a, sizeof(double) * n, cudaMemcpyHostToDevice));
    RR_CUDA(cudaMemcpy(q.b, b, sizeof(double) * n, cudaMemcpyHostToDevice));
    rr::OptState st;
    st.opt = rr::default_adam_options();
    st.lr = st.opt.learning_rate;
    for (int r = 0; r < runs; ++r) {
      const rr_adam_result res = rr::adam_run(st, q);
      energy_best[r] = res.energy_best;
      iterations[r] = res.iterations;
      restart[r] = res.restart_requested;
      rate[r] = res.learning_rate;
    }
    RR_CUDA(cudaMemcpy(x_out, q.x, sizeof(double) * n, cudaMemcpyDeviceToHost));
  });
}

}  // extern "C"
