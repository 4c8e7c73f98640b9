// X2C-HF SCF over a batch of uneven instances in lockstep (the geometry scan run as one program):
// the loop of X2C_HF.cpp:43-138 with the RI Fock build of X2C_FockMatrixRi.cpp:79-205, once per
// iteration for every instance still iterating, each phase one grouped launch:
//
//   c_t from the previous SP2 projector Pi: Y = Pi G, CholeskyQR2 (grouped GEMMs + one Cholesky
//       CTA per instance), c_t = Y^dagger X^dagger
//   J: gamma_P = sum B^P_mn Re(P_aa + P_bb)_mn, J = sum_P gamma_P B^P       (grouped GEMV kernels)
//   K: half-transforms T_f[P] = [Re c_f; Im c_f] B^P and the three exchange blocks (two Hermitian
//       diagonal blocks, the off-diagonal one by Gauss's three products)   (grouped GEMMs)
//   F = h + J - K, E = 1/2 Re Tr[P (h + F)], DIIS on e = F P S - S P F (device dots, host solve)
//   Fo = X^dagger F X, SP2 purification from Gershgorin bounds, P_new = X Pi X^dagger
//       (Kramers-projected), max |P_new - P|
//
// The GEMMs of a phase go through gemm_grouped (one persistent launch per tile configuration over all
// instances' tiles); the elementwise and reduction kernels take a table of per-instance descriptors
// and an active list, with blockIdx.y selecting the instance.  Reductions are fixed-order (GRC partials
// per instance, then one CTA), so every instance computes the same numbers in any batch.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <mutex>
#include <vector>

#include "chol.cuh"
#include "grouped.cuh"
#include "ri_store.cuh"

namespace rr {

namespace {

constexpr int GRC = 32;    // reduction partials per instance
constexpr int GDIIS = 16;  // DIIS vectors at most
constexpr int SCAL = 32;   // scalars per instance: 0 E, 1 dP, 2-3 SP2 traces, 4-5 bounds, 6-7 tr / fro, 8.. dots
// partial-sum layout per instance (doubles)
constexpr int P_E = 0, P_D = GRC, P_S0 = 2 * GRC, P_S1 = 4 * GRC, P_GB = 6 * GRC, P_TF = 8 * GRC, P_DOT = 10 * GRC;
constexpr int P_TOTAL = P_DOT + GDIIS * GRC;

struct GDev {
  int64_t nl, n, ne, r, naux, pitch, nb;
  const double *B, *h, *X, *S;
  double *P, *Pn, *F, *Fs, *e, *PS, *SP, *tmp, *tmp2, *Fo, *Pi, *T2;
  double *Dp, *gam, *J, *Ct, *Cs0, *Cs1, *T0, *T1, *Tm0, *Tp1;
  double *K00r, *K00i, *K11r, *K11i, *K01r, *K01i, *K2;
  double *Gm, *Y2, *Y3, *Mm, *Wt, *PQ;
  double *part, *scal;
  double *err, *val;  // DIIS slots: slot k at + k * 2 n^2
  int* status;
  double coef[GDIIS];
  int32_t ord[GDIIS];
  int32_t ncoef, slot_new, ndots, kramers;
};

__device__ __forceinline__ const GDev& inst(const GDev* tab, const int* act) { return tab[act[blockIdx.y]]; }

__device__ __forceinline__ double gsum(double v) {
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += red[w];
  return t;
}

__device__ __forceinline__ double gmax(double v, bool is_min) {
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = is_min ? fmin(v, w) : fmax(v, w);
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = red[0];
  if (threadIdx.x == 0)
    for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) t = is_min ? fmin(t, red[w]) : fmax(t, red[w]);
  return t;
}

// [beg, end) of this CTA's chunk of cnt items over gridDim.x CTAs
__device__ __forceinline__ void gchunk(int64_t cnt, int64_t& beg, int64_t& end) {
  const int64_t per = (cnt + gridDim.x - 1) / gridDim.x;
  beg = blockIdx.x * per;
  end = beg + per < cnt ? beg + per : cnt;
}

#define GLOOP(i, cnt) \
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < (cnt); i += static_cast<int64_t>(gridDim.x) * blockDim.x)

// ---- Fock build ----

// Dp = Re(P_aa + P_bb) (nl x nl)
__global__ void k_spin_sum(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  const int64_t nl = d.nl, n = d.n;
  GLOOP(idx, nl * nl) {
    const int64_t a = idx / nl, b = idx % nl;
    d.Dp[idx] = d.P[(a * n + b) * 2] + d.P[((nl + a) * n + nl + b) * 2];
  }
}

// gamma_P = sum_k B[P][k] Dp[k], one warp per P
__global__ void k_gamma(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  const int lane = threadIdx.x & 31;
  const int64_t nw = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  const int64_t nn = d.nl * d.nl;
  for (int64_t P = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); P < d.naux; P += nw) {
    const double* b = d.B + P * d.pitch;
    double s = 0.0;
    for (int64_t k = lane; k < nn; k += 32) s = fma(b[k], d.Dp[k], s);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) d.gam[P] = s;
  }
}

// J[k] = sum_P gamma_P B[P][k]
__global__ void k_jmat(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  GLOOP(k, d.nl * d.nl) {
    double s = 0.0;
    for (int64_t P = 0; P < d.naux; ++P) s = fma(d.gam[P], d.B[P * d.pitch + k], s);
    d.J[k] = s;
  }
}

// Cs_f (2r x nl, rows [Re c; Im c]) of the two spin blocks of c_t (r x n complex)
__global__ void k_split(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  const int64_t r = d.r, nl = d.nl, per = 2 * r * nl;
  GLOOP(idx, 2 * per) {
    const int64_t f = idx / per, rem = idx % per, i = rem / nl, a = rem % nl;
    const int64_t ii = i < r ? i : i - r;
    (f == 0 ? d.Cs0 : d.Cs1)[rem] = d.Ct[(ii * d.n + f * nl + a) * 2 + (i < r ? 0 : 1)];
  }
}

// Gauss planes: Tm0 = Re T0 - Im T0, Tp1 = Re T1 + Im T1
__global__ void k_plane_pm(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  const int64_t cnt = d.naux * d.r * d.nl;
  GLOOP(i, cnt) {
    d.Tm0[i] = d.T0[i] - d.T0[cnt + i];
    d.Tp1[i] = d.T1[i] + d.T1[cnt + i];
  }
}

// 3M combine of the off-diagonal block: Re K = P1 + P2, Im K = P3 - P1 + P2
__global__ void k_combine3m(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  GLOOP(i, d.nl * d.nl) {
    const double p1 = d.K01r[i], p2 = d.K2[i];
    d.K01i[i] = d.K01i[i] - p1 + p2;
    d.K01r[i] = p1 + p2;
  }
}

// F = h + G, G = J - K: diagonal blocks -K_ff + J (real part), (0,1) block -K01, (1,0) block -K01^dagger
__global__ void k_fock(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  const int64_t n = d.n, nl = d.nl;
  GLOOP(idx, n * n) {
    const int64_t i = idx / n, j = idx % n;
    double gr, gi;
    if (i < nl && j < nl) {
      gr = -d.K00r[i * nl + j] + d.J[i * nl + j];
      gi = -d.K00i[i * nl + j];
    } else if (i >= nl && j >= nl) {
      const int64_t a = i - nl, b = j - nl;
      gr = -d.K11r[a * nl + b] + d.J[a * nl + b];
      gi = -d.K11i[a * nl + b];
    } else if (i < nl) {
      const int64_t b = j - nl;
      gr = -d.K01r[i * nl + b];
      gi = -d.K01i[i * nl + b];
    } else {
      const int64_t a = i - nl;
      gr = -d.K01r[j * nl + a];
      gi = d.K01i[j * nl + a];
    }
    d.F[2 * idx] = d.h[2 * idx] + gr;
    d.F[2 * idx + 1] = d.h[2 * idx + 1] + gi;
  }
}

// ---- reductions ----

// part[P_E + b] = this CTA's share of sum_ij Re(P_ij (h + F)_ji)
__global__ void k_energy_part(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  const int64_t n = d.n;
  int64_t beg, end;
  gchunk(n * n, beg, end);
  double acc = 0.0;
  for (int64_t idx = beg + threadIdx.x; idx < end; idx += blockDim.x) {
    const int64_t i = idx / n, j = idx % n, t = j * n + i;
    acc += d.P[2 * idx] * (d.h[2 * t] + d.F[2 * t]);
    acc -= d.P[2 * idx + 1] * (d.h[2 * t + 1] + d.F[2 * t + 1]);
  }
  acc = gsum(acc);
  if (threadIdx.x == 0) d.part[P_E + blockIdx.x] = acc;
}

// part[P_D + b] = this CTA's max |Pn - P|
__global__ void k_maxdiff_part(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  int64_t beg, end;
  gchunk(d.n * d.n, beg, end);
  double m = 0.0;
  for (int64_t i = beg + threadIdx.x; i < end; i += blockDim.x)
    m = fmax(m, hypot(d.Pn[2 * i] - d.P[2 * i], d.Pn[2 * i + 1] - d.P[2 * i + 1]));
  m = gmax(m, false);
  if (threadIdx.x == 0) d.part[P_D + blockIdx.x] = m;
}

// part[P_TF + b], part[P_TF + GRC + b]: this CTA's share of Re tr Pi and ||Pi||_F^2 (ne x ne)
__global__ void k_trace_fro_part(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  const int64_t ne = d.ne;
  int64_t beg, end;
  gchunk(ne * ne, beg, end);
  double tr = 0.0, fro = 0.0;
  for (int64_t idx = beg + threadIdx.x; idx < end; idx += blockDim.x) {
    const double re = d.Pi[2 * idx], im = d.Pi[2 * idx + 1];
    fro += re * re + im * im;
    if (idx / ne == idx % ne) tr += re;
  }
  tr = gsum(tr);
  fro = gsum(fro);
  if (threadIdx.x == 0) {
    d.part[P_TF + blockIdx.x] = tr;
    d.part[P_TF + GRC + blockIdx.x] = fro;
  }
}

// scal[out + k] = scale * op over the `cnt` partials part[off + k * stride ...], k < rows (one CTA per
// instance, fixed order); op 0 sum, 1 min, 2 max
template <int OP>
__global__ void k_reduce(const GDev* tab, const int* act, int off, int stride, int cnt, int rows, int out,
                         double scale) {
  const GDev& d = inst(tab, act);
  for (int k = 0; k < rows; ++k) {
    double v = OP == 0 ? 0.0 : (OP == 1 ? 1e300 : -1e300);
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      const double x = d.part[off + k * stride + i];
      v = OP == 0 ? v + x : (OP == 1 ? fmin(v, x) : fmax(v, x));
    }
    const double t = OP == 0 ? gsum(v) : gmax(v, OP == 1);
    if (threadIdx.x == 0) d.scal[out + k] = scale * t;
  }
}

// ---- DIIS ----

__global__ void k_diis_store(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  const int64_t len = 2 * d.n * d.n;
  double* e = d.err + d.slot_new * len;
  double* v = d.val + d.slot_new * len;
  GLOOP(i, len) {
    e[i] = d.e[i];
    v[i] = d.F[i];
  }
}

// part[P_DOT + k GRC + b] = this CTA's share of <err[slot_new], err[ord[k]]>
__global__ void k_diis_dots(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  const int64_t len = 2 * d.n * d.n;
  const double* e = d.err + d.slot_new * len;
  int64_t beg, end;
  gchunk(len, beg, end);
  for (int k = 0; k < d.ndots; ++k) {
    const double* v = d.err + d.ord[k] * len;
    double acc = 0.0;
    for (int64_t i = beg + threadIdx.x; i < end; i += blockDim.x) acc += e[i] * v[i];
    acc = gsum(acc);
    if (threadIdx.x == 0) d.part[P_DOT + k * GRC + blockIdx.x] = acc;
  }
}

// Fs = sum_k coef[k] val[ord[k]], or F when nothing extrapolates (ncoef = 0)
__global__ void k_diis_combine(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  const int64_t len = 2 * d.n * d.n;
  GLOOP(i, len) {
    if (d.ncoef == 0) {
      d.Fs[i] = d.F[i];
    } else {
      double s = 0.0;
      for (int k = 0; k < d.ncoef; ++k) s += d.coef[k] * d.val[d.ord[k] * len + i];
      d.Fs[i] = s;
    }
  }
}

// ---- SP2 ----

// Gershgorin bounds of Fo, a warp per row: part[P_GB + b] = min (a_ii - r_i), part[P_GB + GRC + b] = max
__global__ void k_gersh_part(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  const int64_t n = d.ne;
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  double lo = 1e300, hi = -1e300;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * nw + (threadIdx.x >> 5); i < n;
       i += static_cast<int64_t>(gridDim.x) * nw) {
    double r = 0.0;
    for (int64_t j = lane; j < n; j += 32)
      if (j != i) r += hypot(d.Fo[(i * n + j) * 2], d.Fo[(i * n + j) * 2 + 1]);
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    lo = fmin(lo, d.Fo[(i * n + i) * 2] - r);
    hi = fmax(hi, d.Fo[(i * n + i) * 2] + r);
  }
  lo = gmax(lo, true);
  hi = gmax(hi, false);
  if (threadIdx.x == 0) {
    d.part[P_GB + blockIdx.x] = lo;
    d.part[P_GB + GRC + blockIdx.x] = hi;
  }
}

// X (in Pi) = (emax I - Fo) / (emax - emin) with the partials (tr X, ||X||_F^2) into P_S0
__global__ void k_sp2_init(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  const int64_t n = d.ne;
  const double emin = d.scal[4], emax = d.scal[5], inv = 1.0 / fmax(emax - emin, 1e-300);
  int64_t beg, end;
  gchunk(n * n, beg, end);
  double tr = 0.0, fro = 0.0;
  for (int64_t idx = beg + threadIdx.x; idx < end; idx += blockDim.x) {
    const int64_t i = idx / n, j = idx % n;
    const double re = ((i == j ? emax : 0.0) - d.Fo[2 * idx]) * inv, im = -d.Fo[2 * idx + 1] * inv;
    d.Pi[2 * idx] = re;
    d.Pi[2 * idx + 1] = im;
    fro += re * re + im * im;
    if (i == j) tr += re;
  }
  tr = gsum(tr);
  fro = gsum(fro);
  if (threadIdx.x == 0) {
    d.part[P_S0 + blockIdx.x] = tr;
    d.part[P_S0 + GRC + blockIdx.x] = fro;
  }
}

// Trace-correcting SP2 step on X (Pi) with T2 = X^2 (its upper triangle; the lower one is read as the
// Hermitian mirror): t1 = tr X, t2 = tr X^2 from the partials at pin; X <- X^2 if that brings the trace
// closer to N = r, else 2X - X^2; scal[2..3] = (t1, t2); partials of the new X at pout.
__global__ void k_sp2_step(const GDev* tab, const int* act, int pin, int pout) {
  const GDev& d = inst(tab, act);
  __shared__ int sq;
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < GRC; i += blockDim.x) {
    a += d.part[pin + i];
    b += d.part[pin + GRC + i];
  }
  a = gsum(a);
  b = gsum(b);
  const double N = static_cast<double>(d.r);
  if (threadIdx.x == 0) {
    sq = fabs(b - N) < fabs(2.0 * a - b - N) ? 1 : 0;
    if (blockIdx.x == 0) {
      d.scal[2] = a;
      d.scal[3] = b;
    }
  }
  __syncthreads();
  const bool square = sq != 0;
  const int64_t n = d.ne;
  int64_t beg, end;
  gchunk(n * n, beg, end);
  double tr = 0.0, fro = 0.0;
  for (int64_t idx = beg + threadIdx.x; idx < end; idx += blockDim.x) {
    const int64_t i = idx / n, j = idx % n;
    const int64_t u = i <= j ? idx : j * n + i;
    const double t2[2] = {d.T2[2 * u], i <= j ? d.T2[2 * u + 1] : -d.T2[2 * u + 1]};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const double x = square ? t2[q] : 2.0 * d.Pi[2 * idx + q] - t2[q];
      d.Pi[2 * idx + q] = x;
      fro += x * x;
      if (q == 0 && i == j) tr += x;
    }
  }
  tr = gsum(tr);
  fro = gsum(fro);
  if (threadIdx.x == 0) {
    d.part[pout + blockIdx.x] = tr;
    d.part[pout + GRC + blockIdx.x] = fro;
  }
}

// Time-reversal-even part (X2C [alpha; beta] layout, blocks of nb): Pn = 1/2 (e + s s' conj(e(partner)))
__global__ void k_kramers(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  const int64_t n = d.n, nb = d.nb;
  GLOOP(idx, n * n) {
    const int64_t a = idx / n, b = idx % n;
    const int64_t pa = ((a / nb) ^ 1) * nb + a % nb, pb = ((b / nb) ^ 1) * nb + b % nb;
    const double sg = (((a / nb) % 2 == 0) ? 1.0 : -1.0) * (((b / nb) % 2 == 0) ? 1.0 : -1.0);
    const int64_t q = pa * n + pb;
    d.Pn[2 * idx] = 0.5 * (d.e[2 * idx] + sg * d.e[2 * q]);
    d.Pn[2 * idx + 1] = 0.5 * (d.e[2 * idx + 1] - sg * d.e[2 * q + 1]);
  }
}

// Pn = mix Pn + (1 - mix) P (linear mixing without DIIS)
__global__ void k_mix(const GDev* tab, const int* act, double mix) {
  const GDev& d = inst(tab, act);
  GLOOP(i, 2 * d.n * d.n) d.Pn[i] = mix * d.Pn[i] + (1.0 - mix) * d.P[i];
}

// P = Kramers-even part of the caller's density (copied into e)
__global__ void k_kramers_p(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  const int64_t n = d.n, nb = d.nb;
  GLOOP(idx, n * n) {
    const int64_t a = idx / n, b = idx % n;
    const int64_t pa = ((a / nb) ^ 1) * nb + a % nb, pb = ((b / nb) ^ 1) * nb + b % nb;
    const double sg = (((a / nb) % 2 == 0) ? 1.0 : -1.0) * (((b / nb) % 2 == 0) ? 1.0 : -1.0);
    const int64_t q = pa * n + pb;
    d.P[2 * idx] = 0.5 * (d.e[2 * idx] + sg * d.e[2 * q]);
    d.P[2 * idx + 1] = 0.5 * (d.e[2 * idx + 1] - sg * d.e[2 * q + 1]);
  }
}

// ---- occupied spinors from a projector ----

// The fixed test matrix G (ne x r complex) of the CholeskyQR start: entries in [-1, 1) from a 64-bit
// hash of the index (the single-instance recovery uses the same G).
__global__ void k_fill_gm(const GDev* tab, const int* act) {
  const GDev& d = inst(tab, act);
  GLOOP(idx, 2 * d.ne * d.r) {
    uint64_t z = static_cast<uint64_t>(idx) + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    d.Gm[idx] = static_cast<double>(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
  }
}

// One CTA per instance: Wt = L^{-dagger} (inverse) or L of Mm = L L^dagger (r x r complex), factor and
// inverse in shared memory.
__global__ void __launch_bounds__(CHOL_THREADS) k_chol(const GDev* tab, const int* act, int inverse) {
  extern __shared__ double csm[];
  const GDev& d = tab[act[blockIdx.x]];
  chol_block_body<2>(d.Mm, static_cast<int>(d.r), d.Wt, inverse, d.status, csm);
}

// Occupied count r of the next Fock build, and the places that depend on it: the second spin block's
// split rows and half-transform planes follow the first block's.
void set_rank(GDev& d, int64_t r) {
  d.r = r;
  d.Cs1 = d.Cs0 + 2 * r * d.nl;
  d.T1 = d.T0 + 2 * d.naux * r * d.nl;
}

int gblocks(int64_t per_inst) {
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(64, (per_inst + 255) / 256)));
}

// ------------------------------------------------------------------------------ host side

struct GHost {
  rr_x2c_instance* in = nullptr;
  rr_ri_store* h = nullptr;
  GDev d{};
  double* scal_host = nullptr;  // its row of the gathered scalars
  bool ok = true, active = true, converged = false, grouped_first = false;
  int64_t it = 0;
  double prev = 0.0;
  int maxv = 0;
  std::vector<int> order;
  std::vector<std::vector<double>> bmat;
  std::vector<double> hist;
  int ycur = 0;  // 0: the orthonormal basis is in Y2, 1: in Y3
};

GemmDesc cg(int64_t M, int64_t N, int64_t K, const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
            int64_t ldc) {
  GemmDesc g;
  g.cplx = true;
  g.M = M; g.N = N; g.K = K;
  g.A = A; g.lda = lda; g.B = B; g.ldb = ldb; g.C = C; g.ldc = ldc;
  return g;
}

// Batch-level resources kept per device between calls (a stream, the table space, split-K scratch, the
// gathered scalars), so that a repeated scan allocates nothing; calls on one device take turns.
struct GroupCtx {
  std::mutex mu;
  cudaStream_t s = nullptr;
  TableRing ring;
  DevBuf<double> work, scal_all;
  DevBuf<int> status_all;
  cudaEvent_t ev[4] = {};
};

GroupCtx& group_ctx() {
  static GroupCtx* ctx[kMaxDevices] = {};
  static std::mutex mk;
  const int d = current_device();
  std::lock_guard<std::mutex> lk(mk);
  if (!ctx[d]) {
    auto* c = new GroupCtx();  // kept for the process: its CUDA objects are never released at exit
    RR_CUDA(cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking));
    for (auto& e : c->ev) RR_CUDA(cudaEventCreate(&e));
    c->ring.reserve(size_t{8} << 20);
    ctx[d] = c;
  }
  return *ctx[d];
}

struct Batch {
  GroupCtx& c;
  std::vector<GHost> gs;
  cudaStream_t s;
  TableRing& ring;
  DevBuf<double>& work;
  DevBuf<double>& scal_all;
  DevBuf<int>& status_all;
  std::vector<double> scal_host;
  double wait_ms = 0.0;
  explicit Batch(GroupCtx& ctx)
      : c(ctx), s(ctx.s), ring(ctx.ring), work(ctx.work), scal_all(ctx.scal_all), status_all(ctx.status_all) {}

  // table of every instance's descriptor, as it is now
  const GDev* upload_tab() {
    std::vector<GDev> t(gs.size());
    for (size_t i = 0; i < gs.size(); ++i) t[i] = gs[i].d;
    return static_cast<const GDev*>(ring.put(t.data(), sizeof(GDev) * t.size(), s));
  }
  // (nullptr for an empty list: nothing is launched over it)
  const int* upload_list(const std::vector<int>& a) {
    if (a.empty()) return nullptr;
    return static_cast<const int*>(ring.put(a.data(), sizeof(int) * a.size(), s));
  }
  int64_t max_over(const std::vector<int>& a, int64_t (*f)(const GDev&)) const {
    int64_t m = 1;
    for (int i : a) m = std::max(m, f(gs[i].d));
    return m;
  }
  void sync_scalars() {
    RR_CUDA(cudaMemcpyAsync(scal_host.data(), scal_all.p, sizeof(double) * scal_host.size(), cudaMemcpyDeviceToHost, s));
    const auto w0 = std::chrono::steady_clock::now();
    RR_CUDA(cudaStreamSynchronize(s));
    wait_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
    ring.reset();
  }
  double gemm_ms = 0.0;
  void gemms(const std::vector<GemmDesc>& g) {
    const auto t0 = std::chrono::steady_clock::now();
    gemm_grouped(g, s, ring, work, nullptr);
    gemm_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
};

#define GLAUNCH(kern, gx, nact, ...)                                                      \
  do {                                                                                    \
    if ((nact) > 0) {                                                                     \
      kern<<<dim3(static_cast<unsigned>(gx), static_cast<unsigned>(nact)), 256, 0, b.s>>>(__VA_ARGS__); \
      RR_LAUNCH_CHECK();                                                                  \
    }                                                                                     \
  } while (0)

// c_t (r x n) from the projector in Pi (weighted: F = Q chol(Q^dagger Pi Q), for a start density
// that is a projector only to rounding) for the instances in a.
void grouped_ct(Batch& b, const std::vector<int>& a, bool weighted) {
  if (a.empty()) return;
  const int na = static_cast<int>(a.size());
  const GDev* tab = b.upload_tab();
  const int* al = b.upload_list(a);
  std::vector<GemmDesc> g;
  for (int i : a) {
    const GDev& d = b.gs[i].d;
    g.push_back(cg(d.ne, d.r, d.ne, d.Pi, d.ne, d.Gm, d.r, d.Y2, d.r));
  }
  b.gemms(g);
  int64_t rmax = 1;
  for (int i : a) rmax = std::max(rmax, b.gs[i].d.r);
  const size_t csm = sizeof(double) * static_cast<size_t>(2 * 2 * rmax * (rmax | 1) + rmax);
  RR_REQUIRE(csm <= 227 * 1024, RR_ERR_UNSUPPORTED, "rr_scf_run_x2c_grouped: too many occupied spinors for one CTA");
  static std::atomic<bool> attr[kMaxDevices];
  once_per_device(attr, [] {
    RR_CUDA(cudaFuncSetAttribute(k_chol, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  });
  auto chol = [&](int inverse) {
    k_chol<<<na, CHOL_THREADS, csm, b.s>>>(tab, al, inverse);
    RR_LAUNCH_CHECK();
  };
  for (int i : a) b.gs[i].ycur = 0;
  const int passes = 2;
  for (int pass = 0; pass < passes + (weighted ? 1 : 0); ++pass) {
    const bool wpass = pass == passes;
    g.clear();
    if (wpass) {
      for (int i : a) {
        const GDev& d = b.gs[i].d;
        const double* cur = b.gs[i].ycur ? d.Y3 : d.Y2;
        g.push_back(cg(d.ne, d.r, d.ne, d.Pi, d.ne, cur, d.r, d.PQ, d.r));
      }
      b.gemms(g);
      g.clear();
    }
    for (int i : a) {
      const GDev& d = b.gs[i].d;
      const double* cur = b.gs[i].ycur ? d.Y3 : d.Y2;
      GemmDesc m = cg(d.r, d.r, d.ne, cur, d.r, wpass ? d.PQ : cur, d.r, d.Mm, d.r);
      m.opA = Op::T;
      m.conjA = true;
      g.push_back(m);
    }
    b.gemms(g);
    chol(wpass ? 0 : 1);
    g.clear();
    for (int i : a) {
      const GDev& d = b.gs[i].d;
      const double* cur = b.gs[i].ycur ? d.Y3 : d.Y2;
      double* nxt = b.gs[i].ycur ? d.Y2 : d.Y3;
      g.push_back(cg(d.ne, d.r, d.r, cur, d.r, d.Wt, d.r, nxt, d.r));
    }
    b.gemms(g);
    for (int i : a) b.gs[i].ycur ^= 1;
  }
  g.clear();
  for (int i : a) {
    const GDev& d = b.gs[i].d;
    GemmDesc c = cg(d.r, d.n, d.ne, b.gs[i].ycur ? d.Y3 : d.Y2, d.r, d.X, d.ne, d.Ct, d.n);
    c.opA = Op::T;
    c.conjA = true;
    c.opB = Op::T;
    c.conjB = true;
    g.push_back(c);
  }
  b.gemms(g);
}

}  // namespace

void scf_x2c_grouped(rr_x2c_instance* ins, int64_t count, const rr_scf_opts* so, rr_batch_stats* stats) {
  const auto t0 = std::chrono::steady_clock::now();
  RR_REQUIRE(so->precision == RR_PREC_FP64, RR_ERR_UNSUPPORTED, "rr_scf_run_x2c_grouped: FP64 only");
  RR_REQUIRE(so->max_iterations >= 1, RR_ERR_ARG, "rr_scf_run_x2c_grouped: max_iterations < 1");
  RR_REQUIRE(so->diis_size <= GDIIS, RR_ERR_ARG, "rr_scf_run_x2c_grouped: diis_size too large");
  const bool use_diis = so->diis_size >= 2;
  const bool mixing_on = !use_diis && so->mixing > 0.0 && so->mixing != 1.0;
  GroupCtx& ctx = group_ctx();
  std::lock_guard<std::mutex> ctx_lock(ctx.mu);
  Batch b(ctx);
  b.ring.reset();
  b.gs.resize(static_cast<size_t>(count));
  b.scal_all.ensure(static_cast<size_t>(std::max<int64_t>(count, 1) * SCAL));
  b.status_all.ensure(static_cast<size_t>(std::max<int64_t>(count, 1)));
  RR_CUDA(cudaMemsetAsync(b.status_all.p, 0, sizeof(int) * std::max<int64_t>(count, 1), b.s));
  RR_CUDA(cudaMemsetAsync(b.scal_all.p, 0, sizeof(double) * std::max<int64_t>(count, 1) * SCAL, b.s));
  b.scal_host.assign(static_cast<size_t>(std::max<int64_t>(count, 1) * SCAL), 0.0);
  double tune_s0 = 0.0;
  int64_t tune_l0 = 0;
  autotune_totals(&tune_s0, &tune_l0);
  // kernels launched by this call, without those of the autotuner's timing runs
  auto own_launches = [&] {
    double ts;
    int64_t tl;
    autotune_totals(&ts, &tl);
    return launches() - (tl - tune_l0);
  };
  const int64_t launches0 = own_launches();

  // ---- set-up: validate, allocate, upload ----
  std::vector<int> all;
  for (int64_t i = 0; i < count; ++i) {
    GHost& G = b.gs[i];
    rr_x2c_instance& in = ins[i];
    G.in = &in;
    in.status = RR_OK;
    in.result.electronic_energy = 0.0;
    in.result.iterations = 0;
    in.result.converged = 0;
    in.result.mixed_iterations = 0;
    in.result.fp64_iterations = 0;
    in.result.build_ms = in.result.diis_ms = in.result.density_ms = 0.0;
    try {
      RR_REQUIRE(in.h && in.h_x2c && in.X && in.S && in.P0 && in.P_out, RR_ERR_ARG, "null argument");
      rr_ri_store* h = in.h;
      RR_REQUIRE(h->ntens == 1, RR_ERR_STATE, "handle holds a 4-component store");
      const int64_t nl = h->n, n = 2 * nl, ne = in.n_eff, r = in.n_electrons;
      RR_REQUIRE(ne >= 1 && ne <= n, RR_ERR_ARG, "n_eff out of range");
      RR_REQUIRE(r > 0 && r <= ne, RR_ERR_ARG,
                 "x2cDensityMatrix: n_electrons must be a positive number of spinors that fits within the basis");
      G.h = h;
      const int64_t c2 = 2 * n * n, ce = 2 * n * ne, ee = 2 * ne * ne, naux = h->naux;
      // the occupied count can differ from n_electrons only for a fallback first iteration
      const int64_t rmax = ne;
      Arena ar(&h->scf_buf);  // the handle's SCF buffers, grown on demand and kept between runs
      GDev& d = G.d;
      d.nl = nl; d.n = n; d.ne = ne; d.r = r; d.naux = naux; d.pitch = h->pitch[0]; d.nb = nl;
      d.B = h->B[0].p;
      double *hd, *Xd, *Sd;
      ar.request(&hd, c2);
      ar.request(&Xd, ce);
      ar.request(&Sd, c2);
      ar.request(&d.P, c2);
      ar.request(&d.Pn, c2);
      ar.request(&d.F, c2);
      ar.request(&d.Fs, c2);
      ar.request(&d.e, c2);
      ar.request(&d.PS, c2);
      ar.request(&d.SP, c2);
      ar.request(&d.tmp, std::max(c2, ce));
      ar.request(&d.tmp2, std::max(c2, ce));
      ar.request(&d.Fo, ee);
      ar.request(&d.Pi, ee);
      ar.request(&d.T2, ee);
      ar.request(&d.Dp, nl * nl);
      ar.request(&d.gam, naux);
      ar.request(&d.J, nl * nl);
      ar.request(&d.Ct, 2 * rmax * n);
      ar.request(&d.Cs0, 4 * rmax * nl);         // [Re c_0; Im c_0; Re c_1; Im c_1] (Cs1 follows Cs0)
      ar.request(&d.T0, 4 * naux * rmax * nl);   // the four planes of both half-transforms (T1 follows T0)
      ar.request(&d.Tm0, naux * rmax * nl);
      ar.request(&d.Tp1, naux * rmax * nl);
      for (double** k : {&d.K00r, &d.K00i, &d.K11r, &d.K11i, &d.K01r, &d.K01i, &d.K2}) ar.request(k, nl * nl);
      ar.request(&d.Gm, 2 * ne * rmax);
      ar.request(&d.Y2, 2 * ne * rmax);
      ar.request(&d.Y3, 2 * ne * rmax);
      ar.request(&d.PQ, 2 * ne * rmax);
      ar.request(&d.Mm, 2 * rmax * rmax);
      ar.request(&d.Wt, 2 * rmax * rmax);
      ar.request(&d.part, P_TOTAL);
      const int slots = use_diis ? so->diis_size : 1;
      ar.request(&d.err, slots * c2);
      ar.request(&d.val, slots * c2);
      ar.commit();
      d.h = hd; d.X = Xd; d.S = Sd;
      set_rank(d, r);
      d.scal = b.scal_all.p + i * SCAL;
      d.status = b.status_all.p + i;
      d.kramers = so->kramers_restricted && in.n_electrons % 2 == 0;
      copy_in(hd, in.h_x2c, c2, true, b.s);
      copy_in(Xd, in.X, ce, true, b.s);
      copy_in(Sd, in.S, c2, true, b.s);
      copy_in(d.kramers ? d.e : d.P, in.P0, c2, true, b.s);
      G.scal_host = b.scal_host.data() + i * SCAL;
      G.maxv = use_diis ? so->diis_size : 0;
      G.bmat.assign(static_cast<size_t>(std::max(G.maxv, 1)), std::vector<double>(std::max(G.maxv, 1), 0.0));
      all.push_back(static_cast<int>(i));
    } catch (const Error& e) {
      in.status = e.code;
      G.ok = G.active = false;
    }
  }
  // start densities (Kramers-even part when restricted) and the CholeskyQR test matrices
  {
    std::vector<int> kr;
    for (int i : all)
      if (b.gs[i].d.kramers) kr.push_back(i);
    const GDev* tab = b.upload_tab();
    if (!kr.empty()) {
      const int* kl = b.upload_list(kr);
      GLAUNCH(k_kramers_p, gblocks(b.max_over(kr, [](const GDev& d) { return d.n * d.n; })), kr.size(), tab, kl);
    }
    const int* al = b.upload_list(all);
    GLAUNCH(k_fill_gm, gblocks(b.max_over(all, [](const GDev& d) { return 2 * d.ne * d.r; })), all.size(), tab, al);
  }

  // ---- first iteration's occupied spinors: Pi0 = (S X)^dagger P (S X) ----
  {
    std::vector<GemmDesc> g;
    for (int i : all) {
      const GDev& d = b.gs[i].d;
      g.push_back(cg(d.n, d.ne, d.n, d.S, d.n, d.X, d.ne, d.tmp, d.ne));
    }
    b.gemms(g);
    g.clear();
    for (int i : all) {
      const GDev& d = b.gs[i].d;
      g.push_back(cg(d.n, d.ne, d.n, d.P, d.n, d.tmp, d.ne, d.tmp2, d.ne));
    }
    b.gemms(g);
    g.clear();
    for (int i : all) {
      const GDev& d = b.gs[i].d;
      GemmDesc q = cg(d.ne, d.ne, d.n, d.tmp, d.ne, d.tmp2, d.ne, d.Pi, d.ne);
      q.opA = Op::T;
      q.conjA = true;
      q.mirror = 1;
      g.push_back(q);
    }
    b.gemms(g);
    const GDev* tab = b.upload_tab();
    const int* al = b.upload_list(all);
    GLAUNCH(k_trace_fro_part, GRC, all.size(), tab, al);
    GLAUNCH(k_reduce<0>, 1, all.size(), tab, al, P_TF, GRC, GRC, 2, 6, 1.0);
    b.sync_scalars();
    std::vector<int> grouped, fallback;
    for (int i : all) {
      GHost& G = b.gs[i];
      const double tr = G.scal_host[6], fro = G.scal_host[7], N = static_cast<double>(G.d.r);
      const double tol = 1e-8 * std::max(1.0, N);
      if (std::fabs(tr - N) < tol && std::fabs(fro - tr) < tol) grouped.push_back(i);
      else fallback.push_back(i);
    }
    grouped_ct(b, grouped, true);
    for (int i : grouped) b.gs[i].grouped_first = true;
    for (int i : fallback) {
      GHost& G = b.gs[i];
      try {
        const int64_t r = occupied_ct(G.h, G.d.X, G.d.S, G.d.P, G.d.n, G.d.ne, 1.0, true, true, G.d.Ct, b.s);
        RR_REQUIRE(r <= G.d.ne, RR_ERR_SOLVER, "occupied recovery rank out of range");
        set_rank(G.d, r);
      } catch (const Error& e) {
        G.in->status = e.code;
        G.ok = G.active = false;
      }
    }
  }
  const int64_t launches_setup = own_launches() - launches0;
  int64_t max_iter_launches = 0, lockstep = 0, sp2_max = 0;
  cudaEvent_t* ev = ctx.ev;
  double phase_ms[3] = {0.0, 0.0, 0.0};

  // ---- lockstep iterations ----
  for (int64_t it = 1; it <= so->max_iterations; ++it) {
    std::vector<int> act;
    for (int i : all)
      if (b.gs[i].active) act.push_back(i);
    if (act.empty()) break;
    lockstep = it;
    const int64_t l_it0 = own_launches();
    const int na = static_cast<int>(act.size());
    RR_CUDA(cudaEventRecord(ev[0], b.s));
    if (it > 1) {
      // occupied spinors of the previous iteration's projector (with linear mixing the density is no
      // projector: single-instance recovery from P)
      if (!mixing_on) {
        for (int i : act) set_rank(b.gs[i].d, b.gs[i].in->n_electrons);
        grouped_ct(b, act, false);
      } else {
        for (int i : act) {
          GHost& G = b.gs[i];
          set_rank(G.d, occupied_ct(G.h, G.d.X, G.d.S, G.d.P, G.d.n, G.d.ne, 1.0, true, true, G.d.Ct, b.s));
        }
      }
    }
    const GDev* tab = b.upload_tab();
    const int* al = b.upload_list(act);
    auto mx = [&](int64_t (*f)(const GDev&)) { return gblocks(b.max_over(act, f)); };
    // J
    GLAUNCH(k_spin_sum, mx([](const GDev& d) { return d.nl * d.nl; }), na, tab, al);
    GLAUNCH(k_gamma, std::min<int64_t>(16, (b.max_over(act, [](const GDev& d) { return d.naux; }) + 7) / 8), na, tab, al);
    GLAUNCH(k_jmat, mx([](const GDev& d) { return d.nl * d.nl; }), na, tab, al);
    // K
    GLAUNCH(k_split, mx([](const GDev& d) { return 4 * d.r * d.nl; }), na, tab, al);
    // the half-transforms of the two spin blocks, T_f[P] = [Re c_f; Im c_f] B^P, as two problems per
    // instance (one product of all four row blocks measured slower: its 4r rows fit no skinny tile)
    std::vector<GemmDesc> g;
    for (int i : act) {
      const GDev& d = b.gs[i].d;
      for (int f = 0; f < 2; ++f) {
        GemmDesc ht;
        ht.M = 2 * d.r; ht.N = d.nl; ht.K = d.nl;
        ht.A = f ? d.Cs1 : d.Cs0; ht.lda = d.nl;
        ht.B = d.B; ht.ldb = d.nl; ht.strideB = d.pitch;
        ht.C = f ? d.T1 : d.T0; ht.ldc = d.nl; ht.strideC = d.r * d.nl;
        ht.c_plane_rows = d.r; ht.c_plane_stride = d.naux * d.r * d.nl;
        ht.batch = d.naux;
        g.push_back(ht);
      }
    }
    b.gemms(g);
    GLAUNCH(k_plane_pm, mx([](const GDev& d) { return d.naux * d.r * d.nl; }), na, tab, al);
    auto kprod = [](const GDev& d, const double* A, const double* B, double* C, int64_t K, int mirror, double alpha,
                    double beta) {
      GemmDesc k;
      k.M = d.nl; k.N = d.nl; k.K = K;
      k.opA = Op::T; k.A = A; k.lda = d.nl; k.B = B; k.ldb = d.nl; k.C = C; k.ldc = d.nl;
      k.mirror = mirror; k.alpha = alpha; k.beta = beta;
      return k;
    };
    g.clear();
    for (int i : act) {
      const GDev& d = b.gs[i].d;
      const int64_t kk = d.naux * d.r, pl = kk * d.nl;
      g.push_back(kprod(d, d.T0, d.T0, d.K00r, 2 * kk, 1, 1.0, 0.0));
      g.push_back(kprod(d, d.T1, d.T1, d.K11r, 2 * kk, 1, 1.0, 0.0));
      g.push_back(kprod(d, d.T0, d.T1, d.K01r, kk, 0, 1.0, 0.0));
      g.push_back(kprod(d, d.T0 + pl, d.T1 + pl, d.K2, kk, 0, 1.0, 0.0));
      g.push_back(kprod(d, d.Tm0, d.Tp1, d.K01i, kk, 0, 1.0, 0.0));
    }
    b.gemms(g);
    g.clear();
    for (int i : act) {
      const GDev& d = b.gs[i].d;
      const int64_t pl = d.naux * d.r * d.nl;
      g.push_back(kprod(d, d.T0, d.T0 + pl, d.K00i, d.naux * d.r, -1, 1.0, 0.0));
      g.push_back(kprod(d, d.T1, d.T1 + pl, d.K11i, d.naux * d.r, -1, 1.0, 0.0));
    }
    b.gemms(g);
    g.clear();
    for (int i : act) {
      const GDev& d = b.gs[i].d;
      const int64_t pl = d.naux * d.r * d.nl;
      g.push_back(kprod(d, d.T0 + pl, d.T0, d.K00i, d.naux * d.r, -1, -1.0, 1.0));
      g.push_back(kprod(d, d.T1 + pl, d.T1, d.K11i, d.naux * d.r, -1, -1.0, 1.0));
    }
    b.gemms(g);
    GLAUNCH(k_combine3m, mx([](const GDev& d) { return d.nl * d.nl; }), na, tab, al);
    GLAUNCH(k_fock, mx([](const GDev& d) { return d.n * d.n; }), na, tab, al);
    // energy
    GLAUNCH(k_energy_part, GRC, na, tab, al);
    GLAUNCH(k_reduce<0>, 1, na, tab, al, P_E, GRC, GRC, 1, 0, 0.5);
    RR_CUDA(cudaEventRecord(ev[1], b.s));
    // DIIS
    if (use_diis) {
      g.clear();
      for (int i : act) {
        const GDev& d = b.gs[i].d;
        g.push_back(cg(d.n, d.n, d.n, d.P, d.n, d.S, d.n, d.PS, d.n));
        g.push_back(cg(d.n, d.n, d.n, d.S, d.n, d.P, d.n, d.SP, d.n));
      }
      b.gemms(g);
      g.clear();
      for (int i : act) {
        const GDev& d = b.gs[i].d;
        g.push_back(cg(d.n, d.n, d.n, d.F, d.n, d.PS, d.n, d.e, d.n));
      }
      b.gemms(g);
      g.clear();
      for (int i : act) {
        const GDev& d = b.gs[i].d;
        GemmDesc m = cg(d.n, d.n, d.n, d.SP, d.n, d.F, d.n, d.e, d.n);
        m.alpha = -1.0;
        m.beta = 1.0;
        g.push_back(m);
      }
      b.gemms(g);
      // history slots (newest first), the reference's Diis::push
      for (int i : act) {
        GHost& G = b.gs[i];
        int slot;
        if (static_cast<int>(G.order.size()) < G.maxv) {
          slot = static_cast<int>(G.order.size());
        } else {
          slot = G.order.back();
          G.order.pop_back();
        }
        G.order.insert(G.order.begin(), slot);
        G.d.slot_new = slot;
        G.d.ndots = static_cast<int32_t>(G.order.size());
        for (size_t k = 0; k < G.order.size(); ++k) G.d.ord[k] = G.order[k];
      }
      tab = b.upload_tab();
      GLAUNCH(k_diis_store, mx([](const GDev& d) { return 2 * d.n * d.n; }), na, tab, al);
      GLAUNCH(k_diis_dots, GRC, na, tab, al);
      GLAUNCH(k_reduce<0>, 1, na, tab, al, P_DOT, GRC, GRC, so->diis_size, 8, 1.0);
      b.sync_scalars();
      for (int i : act) {
        GHost& G = b.gs[i];
        const int slot = G.d.slot_new;
        for (size_t k = 0; k < G.order.size(); ++k)
          G.bmat[slot][G.order[k]] = G.bmat[G.order[k]][slot] = G.scal_host[8 + k];
        G.d.ncoef = 0;
        const size_t total = G.order.size();
        for (size_t m = total; m >= 2; --m) {
          double scale = 0.0;
          for (size_t q = 0; q < m; ++q) scale = std::max(scale, G.bmat[G.order[q]][G.order[q]]);
          if (!(scale > 0.0)) break;
          const size_t nn = m + 1;
          std::vector<double> A(nn * nn, 0.0), rhs(nn, 0.0), x;
          for (size_t p = 0; p < m; ++p)
            for (size_t q = 0; q < m; ++q) A[p * nn + q] = G.bmat[G.order[p]][G.order[q]] / scale;
          for (size_t p = 0; p < m; ++p) A[p * nn + m] = A[m * nn + p] = -1.0;
          rhs[m] = -1.0;
          if (!diis_solve(A, rhs, nn, 1e-14, x)) continue;
          G.d.ncoef = static_cast<int32_t>(m);
          for (size_t p = 0; p < m; ++p) {
            G.d.coef[p] = x[p];
            G.d.ord[p] = G.order[p];
          }
          break;
        }
      }
      tab = b.upload_tab();
      al = b.upload_list(act);
    } else {
      for (int i : act) b.gs[i].d.ncoef = 0;
      tab = b.upload_tab();
      al = b.upload_list(act);
    }
    GLAUNCH(k_diis_combine, mx([](const GDev& d) { return 2 * d.n * d.n; }), na, tab, al);
    RR_CUDA(cudaEventRecord(ev[2], b.s));
    // Fo = X^dagger Fs X
    g.clear();
    for (int i : act) {
      const GDev& d = b.gs[i].d;
      g.push_back(cg(d.n, d.ne, d.n, d.Fs, d.n, d.X, d.ne, d.tmp, d.ne));
    }
    b.gemms(g);
    g.clear();
    for (int i : act) {
      const GDev& d = b.gs[i].d;
      GemmDesc q = cg(d.ne, d.ne, d.n, d.X, d.ne, d.tmp, d.ne, d.Fo, d.ne);
      q.opA = Op::T;
      q.conjA = true;
      q.mirror = 1;
      g.push_back(q);
    }
    b.gemms(g);
    // SP2 (lowest r states of Fo) from Gershgorin bounds
    GLAUNCH(k_gersh_part, GRC, na, tab, al);
    GLAUNCH(k_reduce<1>, 1, na, tab, al, P_GB, GRC, GRC, 1, 4, 1.0);
    GLAUNCH(k_reduce<2>, 1, na, tab, al, P_GB + GRC, GRC, GRC, 1, 5, 1.0);
    GLAUNCH(k_sp2_init, GRC, na, tab, al);
    {
      std::vector<int> sp = act;
      const int* spl = al;
      // the same X^2 products every step: built once per stretch between read-backs, then re-launched
      GroupedPlan sq;
      bool sq_valid = false;
      for (int step = 0; step < 120 && !sp.empty(); ++step) {
        sp2_max = std::max<int64_t>(sp2_max, step + 1);
        if (!sq_valid) {
          g.clear();
          for (int i : sp) {
            const GDev& d = b.gs[i].d;
            GemmDesc q = cg(d.ne, d.ne, d.ne, d.Pi, d.ne, d.Pi, d.ne, d.T2, d.ne);
            q.mirror = 2;  // X^2 is Hermitian: upper tiles only, k_sp2_step reads the rest as the mirror
            g.push_back(q);
          }
          const auto t0 = std::chrono::steady_clock::now();
          gemm_grouped_plan(g, b.s, b.ring, b.work, sq);
          b.gemm_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
          sq_valid = true;
        }
        {
          const auto t0 = std::chrono::steady_clock::now();
          gemm_grouped_exec(sq, b.s, nullptr);
          b.gemm_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
        const int pin = (step & 1) ? P_S1 : P_S0, pout = (step & 1) ? P_S0 : P_S1;
        GLAUNCH(k_sp2_step, GRC, sp.size(), tab, spl, pin, pout);
        if (step % 4 == 3) {
          b.sync_scalars();
          tab = b.upload_tab();
          std::vector<int> keep;
          for (int i : sp) {
            const double t1 = b.gs[i].scal_host[2], t2 = b.gs[i].scal_host[3], N = static_cast<double>(b.gs[i].d.r);
            if (!(std::fabs(t1 - t2) < 1e-11 * std::max(1.0, N) && std::fabs(t1 - N) < 1e-6)) keep.push_back(i);
          }
          sp.swap(keep);
          spl = b.upload_list(sp);
          sq_valid = false;  // the read-back reset the table space
        }
      }
      for (int i : sp) {  // no gap at the Fermi level
        GHost& G = b.gs[i];
        G.in->status = RR_ERR_SOLVER;
        G.ok = G.active = false;
      }
      if (!sp.empty()) {
        act.erase(std::remove_if(act.begin(), act.end(), [&](int i) { return !b.gs[i].active; }), act.end());
        if (act.empty()) continue;
      }
    }
    const int na2 = static_cast<int>(act.size());
    tab = b.upload_tab();
    al = b.upload_list(act);
    // P_new = X Pi X^dagger (Kramers-projected)
    g.clear();
    for (int i : act) {
      const GDev& d = b.gs[i].d;
      g.push_back(cg(d.n, d.ne, d.ne, d.X, d.ne, d.Pi, d.ne, d.tmp, d.ne));
    }
    b.gemms(g);
    g.clear();
    for (int i : act) {
      const GDev& d = b.gs[i].d;
      GemmDesc q = cg(d.n, d.n, d.ne, d.tmp, d.ne, d.X, d.ne, d.kramers ? d.e : d.Pn, d.n);
      q.opB = Op::T;
      q.conjB = true;
      q.mirror = 1;
      g.push_back(q);
    }
    b.gemms(g);
    {
      std::vector<int> kr;
      for (int i : act)
        if (b.gs[i].d.kramers) kr.push_back(i);
      if (!kr.empty()) {
        const int* kl = b.upload_list(kr);
        GLAUNCH(k_kramers, gblocks(b.max_over(kr, [](const GDev& d) { return d.n * d.n; })), kr.size(), tab, kl);
      }
    }
    GLAUNCH(k_maxdiff_part, GRC, na2, tab, al);
    GLAUNCH(k_reduce<2>, 1, na2, tab, al, P_D, GRC, GRC, 1, 1, 1.0);
    RR_CUDA(cudaEventRecord(ev[3], b.s));
    b.sync_scalars();
    for (int q = 0; q < 3; ++q) {
      float t = 0.f;
      RR_CUDA(cudaEventElapsedTime(&t, ev[q], ev[q + 1]));
      phase_ms[q] += t;
    }
    max_iter_launches = std::max(max_iter_launches, own_launches() - l_it0);
    // convergence (X2C_HF.cpp:120-134): dP < tolP or dE < tolE from the second iteration
    std::vector<int> mix;
    for (int i : act) {
      GHost& G = b.gs[i];
      const double energy = G.scal_host[0], dP = G.scal_host[1], dE = std::fabs(energy - G.prev);
      G.it = it;
      G.hist.push_back(energy);
      G.in->result.electronic_energy = energy;
      const bool conv = it > 1 && (dP < so->density_tolerance || dE < so->energy_tolerance);
      G.prev = energy;
      if (conv) {
        G.converged = true;
        G.active = false;
        continue;
      }
      if (mixing_on) mix.push_back(i);
    }
    if (!mix.empty()) {
      tab = b.upload_tab();
      const int* ml = b.upload_list(mix);
      GLAUNCH(k_mix, gblocks(b.max_over(mix, [](const GDev& d) { return 2 * d.n * d.n; })), mix.size(), tab, ml,
              so->mixing);
    }
    for (int i : act) {
      GHost& G = b.gs[i];
      if (G.active) std::swap(G.d.P, G.d.Pn);
    }
  }
  RR_CUDA(cudaStreamSynchronize(b.s));
  // ---- outputs ----
  std::vector<int> st(static_cast<size_t>(std::max<int64_t>(count, 1)), 0);
  RR_CUDA(cudaMemcpy(st.data(), b.status_all.p, sizeof(int) * std::max<int64_t>(count, 1), cudaMemcpyDeviceToHost));
  for (int i : all) {
    GHost& G = b.gs[i];
    rr_x2c_instance& in = *G.in;
    if (!G.ok) continue;
    try {
      if (st[i]) throw Error(RR_ERR_SOLVER, "non-positive pivot in the CholeskyQR of the occupied spinors");
      const int64_t c2 = 2 * G.d.n * G.d.n;
      if (in.energy_history)
        for (size_t k = 0; k < G.hist.size(); ++k) in.energy_history[k] = G.hist[k];
      scf_result_outputs(G.h, G.d.Fs, G.d.X, G.d.n, G.d.ne, true, &in.result, true, b.s);
      copy_out(in.P_out, G.d.P, c2, true, b.s);
      RR_CUDA(cudaStreamSynchronize(b.s));
      in.result.iterations = G.it;
      in.result.converged = G.converged ? 1 : 0;
      in.result.fp64_iterations = G.it;
    } catch (const Error& e) {
      in.status = e.code;
    }
  }
  const auto t1 = std::chrono::steady_clock::now();
  const double secs = std::chrono::duration<double>(t1 - t0).count();
  for (int i : all) b.gs[i].in->result.seconds = secs;
  autotune_flush();
  if (stats) {
    stats->iterations = lockstep;
    stats->launches_total = own_launches() - launches0;
    stats->launches_setup = launches_setup;
    stats->launches_max_iteration = max_iter_launches;
    int64_t gf = 0;
    for (int i : all) gf += b.gs[i].grouped_first ? 1 : 0;
    stats->grouped_instances_first = gf;
    stats->seconds = secs;
    double ts;
    int64_t tl;
    autotune_totals(&ts, &tl);
    stats->autotune_seconds = ts - tune_s0;
    stats->autotune_entries = autotune_entries();
    stats->build_ms = phase_ms[0];
    stats->diis_ms = phase_ms[1];
    stats->density_ms = phase_ms[2];
    stats->sp2_steps_max = sp2_max;
    stats->host_wait_ms = b.wait_ms;
    stats->host_gemm_ms = b.gemm_ms;
  }

}

}  // namespace rr
