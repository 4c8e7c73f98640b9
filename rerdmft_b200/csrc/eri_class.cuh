// Thread-per-item McMurchie-Davidson kernels of the integral engine (integrals.cu), templated on the
// angular-momentum class (l_A, l_B | l_C).  The instantiations are spread over several translation units
// (eri_class_*.cu, compiled in parallel), each exporting one dispatch function.
#pragma once

#include <cmath>

#include "ri_store.cuh"

namespace rr {
namespace eri {

constexpr int kMaxL = 6;        // orbital and aux angular momentum (libcint's limit, i functions)
constexpr int kMaxLSum = 18;    // la + lb + lc

// Contracted shell as the kernel sees it: its primitives (coefficients with f(l) folded in) and, per
// Cartesian component, the output function index (-1: not an output) and its scale.
struct DShell {
  double x, y, z;
  int l, nprim, prim0, map0;
};

// Boys function table: F_n(T_k) for T_k = k / 20 (k = 0 .. 720, T_k <= 36) and n = 0 .. kMaxLSum + 6, from
// the power series (boys_eval, integrals.cu).  Between grid points F_n(T) = sum_{j=0}^{6} F_{n+j}(T_k) (T_k - T)^j / j! (dF_n/dT =
// -F_{n+1}) at the nearest T_k (|T - T_k| <= 1/40: the remainder is below 1.3e-15 F_n), then the downward
// recurrence; above T = 36 the asymptotic F_0 and the upward recurrence.
constexpr int kBoysOrders = kMaxLSum + 7;
constexpr int kBoysPoints = 721;
constexpr double kBoysPerUnit = 20.0;

__device__ __forceinline__ double boys_taylor(const double* row, double d) {
  return row[0] + d * (row[1] + d * (1.0 / 2) * (row[2] + d * (1.0 / 3) * (row[3] + d * (1.0 / 4) *
         (row[4] + d * (1.0 / 5) * (row[5] + d * (1.0 / 6) * row[6])))));
}

template <int N>
__device__ __forceinline__ void boys_fixed(double T, const double* tab, double (&F)[N + 1]) {
  const double e = exp(-T);
  if (T >= 36.0) {
    F[0] = 0.5 * sqrt(M_PI / T);
    const double inv2t = 0.5 / T;
#pragma unroll
    for (int n = 0; n < N; ++n) F[n + 1] = ((2 * n + 1) * F[n] - e) * inv2t;
    return;
  }
  const int k = __double2int_rn(T * kBoysPerUnit);
  F[N] = boys_taylor(tab + k * kBoysOrders + N, k / kBoysPerUnit - T);
#pragma unroll
  for (int n = N - 1; n >= 0; --n) F[n] = (2.0 * T * F[n + 1] + e) * (1.0 / (2 * n + 1));
}

// ------------------------------------------------------------------------------------------------
// Thread-per-item kernels for the low angular-momentum classes, where most primitive triples are:
// one thread computes every output of one (orbital shell pair, aux shell), all tables in registers,
// every loop over components and Hermite indices unrolled at compile time.

template <int L>
struct Cart {
  static constexpr int N = (L + 1) * (L + 2) / 2;
};

// Exponent d (0: x, 1: y, 2: z) of Cartesian component k of angular momentum l in libcint's order; a
// plain function, correct whether the compiler folds it or evaluates it at run time.
__host__ __device__ constexpr int cart_comp(int l, int k, int d) {
  int idx = 0;
  for (int a = l; a >= 0; --a)
    for (int b = l - a; b >= 0; --b) {
      if (idx == k) return d == 0 ? a : (d == 1 ? b : l - a - b);
      ++idx;
    }
  return 0;
}

__host__ __device__ constexpr int rix(int t, int u, int v) {
  return (t + u + v) * (t + u + v + 1) * (t + u + v + 2) / 6 + (u + v) * (u + v + 1) / 2 + v;
}

struct ClassArgs {
  const DShell* sh;
  const double* ex;
  const double* co;
  const int* map_fn;
  const double* map_sc;
  const int2* pairs;  // (A, B) with l_A >= l_B
  int64_t npairs;
  const int* cidx;    // aux shells of the class's l
  int64_t ncs;
  int64_t n;
  double* out;
  const double* boys;
  int metric;  // 1: pairs are (A, the constant function), out = (P|Q) (n x n), items with C < A skipped
};

// E^ab of one dimension for the compile-time (LA, LB): E[i][j][t].
template <int LA, int LB>
__device__ __forceinline__ void e_fixed(double (&E)[LA + 1][LB + 1][LA + LB + 1], double inv2p, double xpa,
                                       double xpb) {
#pragma unroll
  for (int i = 0; i <= LA; ++i)
#pragma unroll
    for (int j = 0; j <= LB; ++j)
#pragma unroll
      for (int t = 0; t <= LA + LB; ++t) {
        double v;
        if (i == 0 && j == 0) {
          v = t == 0 ? 1.0 : 0.0;
        } else if (t > i + j) {
          v = 0.0;
        } else if (i > 0) {
          v = xpa * E[i - 1][j][t];
          if (t > 0) v += inv2p * E[i - 1][j][t - 1];
          if (t + 1 <= i + j - 1) v += (t + 1) * E[i - 1][j][t + 1];
        } else {
          v = xpb * E[i][j - 1][t];
          if (t > 0) v += inv2p * E[i][j - 1][t - 1];
          if (t + 1 <= i + j - 1) v += (t + 1) * E[i][j - 1][t + 1];
        }
        E[i][j][t] = v;
      }
}

__host__ __device__ constexpr int n_herm(int l) { return (l + 1) * (l + 2) * (l + 3) / 6; }

// acc[(ia NB + ib) STRIDE] += w (a b | component IC of c) for one primitive triple, from the E tables of the
// pair, the Hermite Coulomb integrals R and the aux factor's Hermite coefficients Ec; every index is a
// compile-time constant.
template <int LA, int LB, int LC, int IC, int STRIDE>
__device__ __forceinline__ void accum_comp(double* acc, const double (&E)[3][LA + 1][LB + 1][LA + LB + 1],
                                           const double (&R)[n_herm(LA + LB + LC)],
                                           const double (&Ec)[LC + 1][LC + 1], double w) {
  constexpr int NA = Cart<LA>::N, NB = Cart<LB>::N, LAB = LA + LB;
  constexpr int cx = cart_comp(LC, IC, 0), cy = cart_comp(LC, IC, 1), cz = cart_comp(LC, IC, 2);
  double G[n_herm(LAB)];
#pragma unroll
  for (int sl = 0; sl <= LAB; ++sl)
#pragma unroll
    for (int m = 0; m <= sl; ++m)
#pragma unroll
      for (int v = 0; v <= m; ++v) {
        const int u = m - v, t = sl - m;
        double g = 0.0;
#pragma unroll
        for (int tau = cx & 1; tau <= cx; tau += 2)
#pragma unroll
          for (int nu = cy & 1; nu <= cy; nu += 2)
#pragma unroll
            for (int phi = cz & 1; phi <= cz; phi += 2) {
              const double ec = Ec[cx][tau] * Ec[cy][nu] * Ec[cz][phi];
              const double r = R[rix(t + tau, u + nu, v + phi)];
              g += ((tau + nu + phi) & 1) ? -ec * r : ec * r;
            }
        G[rix(t, u, v)] = g;
      }
#pragma unroll
  for (int ia = 0; ia < NA; ++ia)
#pragma unroll
    for (int ib = 0; ib < NB; ++ib) {
      const int ax = cart_comp(LA, ia, 0), ay = cart_comp(LA, ia, 1), az = cart_comp(LA, ia, 2);
      const int bx = cart_comp(LB, ib, 0), by = cart_comp(LB, ib, 1), bz = cart_comp(LB, ib, 2);
      double val = 0.0;
#pragma unroll
      for (int t = 0; t <= ax + bx; ++t)
#pragma unroll
        for (int u = 0; u <= ay + by; ++u)
#pragma unroll
          for (int v = 0; v <= az + bz; ++v)
            val += E[0][ax][bx][t] * E[1][ay][by][u] * E[2][az][bz][v] * G[rix(t, u, v)];
      acc[(ia * NB + ib) * STRIDE] += w * val;
    }
}

// Every component, acc[(ia NB + ib) NC + ic].
template <int LA, int LB, int LC, int IC>
__device__ __forceinline__ void comp_all(double* acc, const double (&E)[3][LA + 1][LB + 1][LA + LB + 1],
                                         const double (&R)[n_herm(LA + LB + LC)],
                                         const double (&Ec)[LC + 1][LC + 1], double w) {
  if constexpr (IC < Cart<LC>::N) {
    accum_comp<LA, LB, LC, IC, Cart<LC>::N>(acc + IC, E, R, Ec, w);
    comp_all<LA, LB, LC, IC + 1>(acc, E, R, Ec, w);
  }
}

// The thread's one component `ic`, acc[ia NB + ib].
template <int LA, int LB, int LC, int IC>
__device__ __forceinline__ void comp_dispatch(int ic, double* acc, const double (&E)[3][LA + 1][LB + 1][LA + LB + 1],
                                              const double (&R)[n_herm(LA + LB + LC)],
                                              const double (&Ec)[LC + 1][LC + 1], double w) {
  if constexpr (IC < Cart<LC>::N) {
    if (ic == IC)
      accum_comp<LA, LB, LC, IC, 1>(acc, E, R, Ec, w);
    else
      comp_dispatch<LA, LB, LC, IC + 1>(ic, acc, E, R, Ec, w);
  }
}

// SPLIT: one thread per (pair, aux shell, aux component) for the classes with many outputs; the component
// is selected among compile-time branches, so every table index stays static.
template <int LA, int LB, int LC, bool SPLIT>
__global__ void __launch_bounds__(128) eri_class_kernel(ClassArgs a) {
  constexpr int NA = Cart<LA>::N, NB = Cart<LB>::N, NC = Cart<LC>::N, NCA = SPLIT ? 1 : NC;
  constexpr int LAB = LA + LB, L = LAB + LC;
  constexpr int NR = n_herm(L);
  const double two_pi25 = 2.0 * M_PI * M_PI * sqrt(M_PI);
  const int64_t total = a.npairs * a.ncs * (SPLIT ? NC : 1);
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int2 pr = a.pairs[idx % a.npairs];
    const int64_t rest = idx / a.npairs;
    const int icsel = SPLIT ? static_cast<int>(rest % NC) : 0;
    const int csh = a.cidx[SPLIT ? rest / NC : rest];
    if (a.metric && csh < pr.x) continue;  // (P|Q) for Q >= P only
    const DShell A = a.sh[pr.x], B = a.sh[pr.y], C = a.sh[csh];
    double acc[NA * NB * NCA];
#pragma unroll
    for (int q = 0; q < NA * NB * NCA; ++q) acc[q] = 0.0;
    const double ab[3] = {A.x - B.x, A.y - B.y, A.z - B.z};
    const double ab2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
    for (int i = 0; i < A.nprim; ++i) {
      const double al = a.ex[A.prim0 + i], cA = a.co[A.prim0 + i];
      for (int j = 0; j < B.nprim; ++j) {
        const double be = a.ex[B.prim0 + j], cB = a.co[B.prim0 + j];
        const double p = al + be, ip = 1.0 / p;
        const double P[3] = {(al * A.x + be * B.x) * ip, (al * A.y + be * B.y) * ip, (al * A.z + be * B.z) * ip};
        const double K = exp(-al * be * ip * ab2);
        double E[3][LA + 1][LB + 1][LAB + 1];
#pragma unroll
        for (int d = 0; d < 3; ++d) e_fixed<LA, LB>(E[d], 0.5 * ip, -be * ip * ab[d], al * ip * ab[d]);
        for (int k = 0; k < C.nprim; ++k) {
          const double ga = a.ex[C.prim0 + k], cC = a.co[C.prim0 + k];
          const double alpha = p * ga / (p + ga);
          const double X = P[0] - C.x, Y = P[1] - C.y, Z = P[2] - C.z;
          double F[L + 1];
          boys_fixed<L>(alpha * (X * X + Y * Y + Z * Z), a.boys, F);
          double pw[L + 1];
          pw[0] = 1.0;
#pragma unroll
          for (int n = 1; n <= L; ++n) pw[n] = pw[n - 1] * (-2.0 * alpha);
          double R[NR];
          R[0] = pw[L] * F[L];
#pragma unroll
          for (int n = L - 1; n >= 0; --n) {
#pragma unroll
            for (int sl = L - n; sl >= 1; --sl)
#pragma unroll
              for (int m = 0; m <= sl; ++m)
#pragma unroll
                for (int v = 0; v <= m; ++v) {
                  const int u = m - v, t = sl - m;
                  double val;
                  if (t > 0) {
                    val = X * R[rix(t - 1, u, v)];
                    if (t > 1) val += (t - 1) * R[rix(t - 2, u, v)];
                  } else if (u > 0) {
                    val = Y * R[rix(t, u - 1, v)];
                    if (u > 1) val += (u - 1) * R[rix(t, u - 2, v)];
                  } else {
                    val = Z * R[rix(t, u, v - 1)];
                    if (v > 1) val += (v - 1) * R[rix(t, u, v - 2)];
                  }
                  R[rix(t, u, v)] = val;
                }
            R[0] = pw[n] * F[n];
          }
          // single-centre Hermite coefficients of the aux factor, Ec[i][t] (t = i, i - 2, ...)
          double Ec[LC + 1][LC + 1];
          const double inv2q = 0.5 / ga;
#pragma unroll
          for (int ii = 0; ii <= LC; ++ii)
#pragma unroll
            for (int t = 0; t <= LC; ++t) {
              double v = 0.0;
              if (ii == 0) {
                v = t == 0 ? 1.0 : 0.0;
              } else {
                if (t > 0) v += inv2q * Ec[ii - 1][t - 1];
                if (t + 1 <= LC) v += (t + 1) * Ec[ii - 1][t + 1];
              }
              Ec[ii][t] = v;
            }
          const double w = cA * cB * cC * two_pi25 / (p * ga * sqrt(p + ga)) * K;
          if constexpr (SPLIT) {
            comp_dispatch<LA, LB, LC, 0>(icsel, acc, E, R, Ec, w);
          } else {
            comp_all<LA, LB, LC, 0>(acc, E, R, Ec, w);
          }
        }
      }
    }
    if (a.metric) {  // B is the constant function (l_B = 0): out[P][Q] and out[Q][P]
      const bool same = csh == pr.x;
#pragma unroll
      for (int ia = 0; ia < NA; ++ia)
#pragma unroll
        for (int ic = 0; ic < NC; ++ic) {
          if (SPLIT && ic != icsel) continue;
          if (same && ia > ic) continue;
          const int fa = a.map_fn[A.map0 + ia], fc = a.map_fn[C.map0 + ic];
          if (fa < 0 || fc < 0) continue;
          const double v = acc[ia * NB * NCA + (SPLIT ? 0 : ic)] * a.map_sc[A.map0 + ia] * a.map_sc[C.map0 + ic];
          a.out[static_cast<int64_t>(fa) * a.n + fc] = v;
          a.out[static_cast<int64_t>(fc) * a.n + fa] = v;
        }
      continue;
    }
    const bool sym = pr.x == pr.y;
#pragma unroll
    for (int ia = 0; ia < NA; ++ia)
#pragma unroll
      for (int ib = 0; ib < NB; ++ib) {
        if (sym && ia > ib) continue;
        const int fa = a.map_fn[A.map0 + ia], fb = a.map_fn[B.map0 + ib];
        if (fa < 0 || fb < 0) continue;
        const double sab = a.map_sc[A.map0 + ia] * a.map_sc[B.map0 + ib];
#pragma unroll
        for (int ic = 0; ic < NC; ++ic) {
          if (SPLIT && ic != icsel) continue;  // ic compile-time, icsel the thread's component
          const int fc = a.map_fn[C.map0 + ic];
          if (fc < 0) continue;
          const double v = acc[(ia * NB + ib) * NCA + (SPLIT ? 0 : ic)] * sab * a.map_sc[C.map0 + ic];
          const int64_t row = static_cast<int64_t>(fc) * a.n * a.n;
          a.out[row + static_cast<int64_t>(fa) * a.n + fb] = v;
          a.out[row + static_cast<int64_t>(fb) * a.n + fa] = v;
        }
      }
  }
}

// Launch of one class kernel (grid-stride, 8 waves of the occupancy at most).  The classes with such a
// kernel (l_A >= l_B, aux l <= 3): one thread per item for the s and p pairs with aux s .. f, (pp| s, p)
// and (ds| s, p); one thread per aux component for (pp| d, f), (ds| d, f) and (dp| s, p, d).  The rest
// take the warp kernel of integrals.cu: (dd| ...), l >= 3, and (dp| f), whose template alone compiled for
// 9 minutes (1.35 of the 12.2 ms of the (H2O)_8 / cc-pVDZ raw tensor ran there before the dp templates).
template <int LA, int LB, int LC, bool SPLIT>
void launch_class(const ClassArgs& a, cudaStream_t s) {
  auto kern = eri_class_kernel<LA, LB, LC, SPLIT>;
  static int per_sm[kMaxDevices] = {};
  const int dev = current_device();
  if (!per_sm[dev]) RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[dev], kern, 128, 0));
  int sms = 0;
  RR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int64_t total = a.npairs * a.ncs * (SPLIT ? Cart<LC>::N : 1);
  const int grid = static_cast<int>(std::max<int64_t>(
      1, std::min<int64_t>((total + 127) / 128, static_cast<int64_t>(sms) * std::max(per_sm[dev], 1) * 8)));
  kern<<<grid, 128, 0, s>>>(a);
  RR_LAUNCH_CHECK();
}

// Dispatchers, one per translation unit: launch the class kernel of (la, lb, lc) when that unit holds it.
bool launch_class_sp(int la, int lb, int lc, const ClassArgs& a, cudaStream_t s);     // eri_class_sp.cu
bool launch_class_split(int la, int lb, int lc, const ClassArgs& a, cudaStream_t s);  // eri_class_split.cu
bool launch_class_dp01(int la, int lb, int lc, const ClassArgs& a, cudaStream_t s);   // eri_class_dp01.cu
bool launch_class_dp2(int la, int lb, int lc, const ClassArgs& a, cudaStream_t s);    // eri_class_dp2.cu

}  // namespace eri
}  // namespace rr
