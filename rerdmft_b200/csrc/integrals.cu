// Two- and three-centre electron-repulsion integrals over contracted Cartesian Gaussians on the GPU:
// the aux metric (P|Q) (reference: auxMetric, src/AO_ints/ThreeCenterIntegrals.cpp:140-161, libcint
// cint2c2e_cart per aux shell pair) and the raw tensor raw[P, p n + q] = (pq|P) (threeCenterIntegralsRaw,
// :163-184, cint3c2e_cart per orbital function pair and aux shell), plus the device set-up of a resident
// RI handle from a basis (riThreeCenterTensor, :219-236, with auxMetricOrthogonalization, :185-189).
//
// Method: McMurchie-Davidson Hermite expansion (J. Comput. Phys. 26, 218 (1978)).  For primitives
// a (exponent alpha, centre A), b (beta, B) and an aux primitive c (gamma, C):
//   (ab|c) = 2 pi^(5/2) / (p gamma sqrt(p + gamma)) K_AB
//            sum_tuv E^ab_t E^ab_u E^ab_v sum_{tau nu phi} (-1)^(tau+nu+phi) E^c_tau E^c_nu E^c_phi
//            R_{t+tau, u+nu, v+phi}(p gamma / (p + gamma), P - C)
// with p = alpha + beta, P = (alpha A + beta B) / p, K_AB = exp(-alpha beta / p |A - B|^2), E the
// Hermite expansion coefficients of each Cartesian factor and R the Hermite Coulomb integrals from the
// Boys function.  The two-centre metric is the same sum with b the constant function 1 (beta = 0).
// Coefficients follow libcint's convention, so the integrals match what the reference's libcint calls
// return for the same basis-function lists: a function is coefficient * f(l) * x^lx y^ly z^lz exp(-a r^2)
// with f(0) = 1/sqrt(4 pi), f(1) = sqrt(3/(4 pi)) and f(l >= 2) = 1.
//
// GPU mapping.  Work items are (orbital shell pair, aux shell), grouped by angular-momentum class
// (l_A >= l_B after swapping the pair).  The low classes, where most primitive triples are (s and p pairs
// with long contractions), run one thread per item (or per item and aux component) in kernels templated
// on (l_A, l_B, l_C): E, R and the accumulators in registers, every component and Hermite loop unrolled.
// The other classes and the metric run one warp per item: per primitive pair lanes 0-2 build the three E
// tables in shared memory; per aux primitive lane 3 evaluates the Boys function and the warp builds the R
// table level by level (in place, one __syncwarp per level); each lane then accumulates its share of the
// (component a, component b, component c) outputs, in chunks of 32 x kOutPerLane.  The Boys function
// comes from a table of F_n at T = k/20 and a 7-term Taylor step.  Every output element is written exactly
// once (both halves of the (pq) symmetry from one value), so nothing is zeroed.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "eri_class.cuh"
#include "ri_store.cuh"

namespace rr {
namespace {

using namespace eri;

constexpr int kOutPerLane = 8;  // accumulators per lane per chunk
constexpr int kIntThreads = 128;


struct IntArgs {
  const DShell* sh;
  const double* ex;
  const double* co;
  const int* map_fn;
  const double* map_sc;
  const int2* pairs;   // bra shell pairs (A, B); B = the unit shell for the metric
  int64_t npairs;
  const int* cidx;     // ket shells
  int64_t nc;
  int metric;          // 1: (A|C) with C >= A, out = M (naux x naux); 0: (AB|C), out = raw (naux x n^2)
  int64_t n;           // orbital function count (raw) or aux count (metric)
  double* out;
  const double* boys;  // Boys function table (boys_table)
  int la_max, lab_max, lc_max, L_max;  // shared-memory sizing
};

__host__ __device__ inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// (lx, ly, lz) of component k of angular momentum l in libcint's order (x-major, then y).
__device__ inline void cart_of(int l, int k, int& lx, int& ly, int& lz) {
  int idx = 0;
  for (int x = l; x >= 0; --x)
    for (int y = l - x; y >= 0; --y) {
      if (idx == k) {
        lx = x;
        ly = y;
        lz = l - x - y;
        return;
      }
      ++idx;
    }
  lx = ly = lz = 0;
}

__device__ inline int r_index(int t, int u, int v) {
  const int s = t + u + v, m = u + v;
  return s * (s + 1) * (s + 2) / 6 + m * (m + 1) / 2 + v;
}

// F_n(T) = int_0^1 t^(2n) exp(-T t^2) dt for n = 0..nmax.  T <= 36: F_nmax from its power series
// exp(-T) sum_k (2T)^k / ((2 nmax + 1)(2 nmax + 3)...(2 nmax + 2k + 1)) (all terms positive), then the
// downward recurrence F_n = (2T F_{n+1} + exp(-T)) / (2n + 1); T > 36: F_0 = sqrt(pi / T) / 2 (erf(sqrt T)
// is 1 to double precision there) and the upward recurrence F_{n+1} = ((2n + 1) F_n - exp(-T)) / (2T),
// stable for T > nmax.
__device__ void boys_eval(int nmax, double T, double* F) {
  const double e = exp(-T);
  if (T > 36.0) {
    F[0] = 0.5 * sqrt(M_PI / T);
    const double inv2t = 0.5 / T;
    for (int n = 0; n < nmax; ++n) F[n + 1] = ((2 * n + 1) * F[n] - e) * inv2t;
    return;
  }
  double term = 1.0 / (2 * nmax + 1), sum = term;
  for (int k = 1; k < 400; ++k) {
    term *= 2.0 * T / (2 * nmax + 2 * k + 1);
    sum += term;
    if (term < 1e-17 * sum) break;
  }
  F[nmax] = e * sum;
  for (int n = nmax - 1; n >= 0; --n) F[n] = (2.0 * T * F[n + 1] + e) / (2 * n + 1);
}


__global__ void boys_table_kernel(double* tab) {
  double F[kBoysOrders];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < kBoysPoints; k += gridDim.x * blockDim.x) {
    boys_eval(kBoysOrders - 1, k / kBoysPerUnit, F);
    for (int n = 0; n < kBoysOrders; ++n) tab[k * kBoysOrders + n] = F[n];
  }
}


__device__ void boys_table_eval(int nmax, double T, const double* tab, double* F) {
  const double e = exp(-T);
  if (T >= 36.0) {
    F[0] = 0.5 * sqrt(M_PI / T);
    const double inv2t = 0.5 / T;
    for (int n = 0; n < nmax; ++n) F[n + 1] = ((2 * n + 1) * F[n] - e) * inv2t;
    return;
  }
  const int k = __double2int_rn(T * kBoysPerUnit);
  F[nmax] = boys_taylor(tab + k * kBoysOrders + nmax, k / kBoysPerUnit - T);
  for (int n = nmax - 1; n >= 0; --n) F[n] = (2.0 * T * F[n + 1] + e) / (2 * n + 1);
}


// E[i][j][t] (flat ((i (lb+1) + j) (la+lb+1) + t)) of one dimension, without K_AB.
__device__ void e_table(double* E, int la, int lb, double p, double xpa, double xpb) {
  const int lt = la + lb + 1;
  const double inv2p = 0.5 / p;
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j) {
      double* dst = E + (i * (lb + 1) + j) * lt;
      if (i == 0 && j == 0) {
        dst[0] = 1.0;
        for (int t = 1; t < lt; ++t) dst[t] = 0.0;
        continue;
      }
      const double* src = i > 0 ? E + ((i - 1) * (lb + 1) + j) * lt : E + (i * (lb + 1) + j - 1) * lt;
      const double x = i > 0 ? xpa : xpb;
      const int top = i + j;  // entries of src beyond i + j - 1 are zero
      for (int t = 0; t < lt; ++t) {
        double v = 0.0;
        if (t <= top) {
          v = x * src[t];
          if (t > 0) v += inv2p * src[t - 1];
          if (t + 1 <= top - 1) v += (t + 1) * src[t + 1];
        }
        dst[t] = v;
      }
    }
}

__global__ void __launch_bounds__(kIntThreads) eri_kernel(IntArgs a) {
  extern __shared__ double smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int esz = (a.la_max + 1) * (a.la_max + 1) * (a.lab_max + 1);  // per dimension, la, lb <= la_max
  const int csz = (a.lc_max + 1) * (a.lc_max + 1);
  const int rsz = (a.L_max + 1) * (a.L_max + 2) * (a.L_max + 3) / 6;
  const int per_warp = 3 * esz + csz + rsz + (a.L_max + 1);
  double* Ex = smem + static_cast<int64_t>(warp) * per_warp;
  double* Ey = Ex + esz;
  double* Ez = Ey + esz;
  double* Ec = Ez + esz;
  double* R = Ec + csz;
  double* F = R + rsz;
  const double two_pi25 = 2.0 * M_PI * M_PI * sqrt(M_PI);

  const int64_t items = a.npairs * a.nc;
  for (int64_t item = static_cast<int64_t>(blockIdx.x) * nwarp + warp; item < items;
       item += static_cast<int64_t>(gridDim.x) * nwarp) {
    const int2 pr = a.pairs[item / a.nc];
    const int ic_sh = a.cidx[item % a.nc];
    if (a.metric && ic_sh < pr.x) continue;  // (P|Q) for Q >= P only
    const DShell A = a.sh[pr.x], B = a.sh[pr.y], C = a.sh[ic_sh];
    const bool sym = a.metric ? (ic_sh == pr.x) : (pr.x == pr.y);
    const int nA = ncart(A.l), nB = ncart(B.l), nCc = ncart(C.l);
    const int nout = nA * nB * nCc;
    const int lab = A.l + B.l, L = lab + C.l;
    const double abx = A.x - B.x, aby = A.y - B.y, abz = A.z - B.z;
    const double ab2 = abx * abx + aby * aby + abz * abz;
    for (int o0 = 0; o0 < nout; o0 += 32 * kOutPerLane) {
      double acc[kOutPerLane];
#pragma unroll
      for (int q = 0; q < kOutPerLane; ++q) acc[q] = 0.0;
      for (int i = 0; i < A.nprim; ++i) {
        const double al = a.ex[A.prim0 + i], ca = a.co[A.prim0 + i];
        for (int j = 0; j < B.nprim; ++j) {
          const double be = a.ex[B.prim0 + j], cb = a.co[B.prim0 + j];
          const double p = al + be;
          const double Px = (al * A.x + be * B.x) / p, Py = (al * A.y + be * B.y) / p, Pz = (al * A.z + be * B.z) / p;
          const double K = exp(-al * be / p * ab2);
          __syncwarp();
          if (lane == 0) e_table(Ex, A.l, B.l, p, -be / p * abx, al / p * abx);
          if (lane == 1) e_table(Ey, A.l, B.l, p, -be / p * aby, al / p * aby);
          if (lane == 2) e_table(Ez, A.l, B.l, p, -be / p * abz, al / p * abz);
          for (int k = 0; k < C.nprim; ++k) {
            const double ga = a.ex[C.prim0 + k], cc = a.co[C.prim0 + k];
            const double alpha = p * ga / (p + ga);
            const double X = Px - C.x, Y = Py - C.y, Z = Pz - C.z;
            __syncwarp();
            if (lane == 3) boys_table_eval(L, alpha * (X * X + Y * Y + Z * Z), a.boys, F);
            if (lane == 4) {  // single-centre Hermite expansion of the aux factor: Ec[i][t]
              const double inv2q = 0.5 / ga;
              for (int ii = 0; ii <= C.l; ++ii)
                for (int t = 0; t <= C.l; ++t) {
                  double v;
                  if (ii == 0) {
                    v = t == 0 ? 1.0 : 0.0;
                  } else {
                    const double* src = Ec + (ii - 1) * (C.l + 1);
                    v = 0.0;
                    if (t > 0) v += inv2q * src[t - 1];
                    if (t + 1 <= C.l) v += (t + 1) * src[t + 1];
                  }
                  Ec[ii * (C.l + 1) + t] = v;
                }
            }
            __syncwarp();
            // R^(n) for n = L .. 0, in place: level s of step n reads levels s - 1, s - 2 of step n + 1
            double m2a = 1.0;
            for (int n = 0; n < L; ++n) m2a *= -2.0 * alpha;  // (-2 alpha)^L
            if (lane == 0) R[0] = m2a * F[L];
            for (int n = L - 1; n >= 0; --n) {
              m2a /= -2.0 * alpha;
              __syncwarp();
              for (int s = L - n; s >= 1; --s) {
                const int cnt = (s + 1) * (s + 2) / 2;
                for (int e = lane; e < cnt; e += 32) {
                  int m = 0;
                  while ((m + 1) * (m + 2) / 2 <= e) ++m;
                  const int v = e - m * (m + 1) / 2, u = m - v, t = s - m;
                  double val;
                  if (t > 0) {
                    val = X * R[r_index(t - 1, u, v)];
                    if (t > 1) val += (t - 1) * R[r_index(t - 2, u, v)];
                  } else if (u > 0) {
                    val = Y * R[r_index(t, u - 1, v)];
                    if (u > 1) val += (u - 1) * R[r_index(t, u - 2, v)];
                  } else {
                    val = Z * R[r_index(t, u, v - 1)];
                    if (v > 1) val += (v - 1) * R[r_index(t, u, v - 2)];
                  }
                  R[r_index(t, u, v)] = val;
                }
                __syncwarp();
              }
              if (lane == 0) R[0] = m2a * F[n];
            }
            __syncwarp();
            const double w = ca * cb * cc * two_pi25 / (p * ga * sqrt(p + ga)) * K;
            const int lt = lab + 1;
#pragma unroll
            for (int q = 0; q < kOutPerLane; ++q) {
              const int o = o0 + q * 32 + lane;
              if (o >= nout) break;
              const int ia = o / (nB * nCc), ib = (o / nCc) % nB, icc = o % nCc;
              int ax, ay, az, bx, by, bz, cx, cy, cz;
              cart_of(A.l, ia, ax, ay, az);
              cart_of(B.l, ib, bx, by, bz);
              cart_of(C.l, icc, cx, cy, cz);
              const double* ex = Ex + (ax * (B.l + 1) + bx) * lt;
              const double* ey = Ey + (ay * (B.l + 1) + by) * lt;
              const double* ez = Ez + (az * (B.l + 1) + bz) * lt;
              double val = 0.0;
              for (int t = 0; t <= ax + bx; ++t)
                for (int u = 0; u <= ay + by; ++u) {
                  const double exy = ex[t] * ey[u];
                  for (int v = 0; v <= az + bz; ++v) {
                    double g = 0.0;
                    for (int tau = cx & 1; tau <= cx; tau += 2)
                      for (int nu = cy & 1; nu <= cy; nu += 2)
                        for (int phi = cz & 1; phi <= cz; phi += 2) {
                          const double ec = Ec[cx * (C.l + 1) + tau] * Ec[cy * (C.l + 1) + nu] *
                                            Ec[cz * (C.l + 1) + phi];
                          const double r = R[r_index(t + tau, u + nu, v + phi)];
                          g += ((tau + nu + phi) & 1) ? -ec * r : ec * r;
                        }
                    val += exy * ez[v] * g;
                  }
                }
              acc[q] += w * val;
            }
          }
        }
      }
#pragma unroll
      for (int q = 0; q < kOutPerLane; ++q) {
        const int o = o0 + q * 32 + lane;
        if (o >= nout) break;
        const int ia = o / (nB * nCc), ib = (o / nCc) % nB, icc = o % nCc;
        const int fa = a.map_fn[A.map0 + ia], fc = a.map_fn[C.map0 + icc];
        if (a.metric) {
          if (fa < 0 || fc < 0 || (sym && ia > icc)) continue;
          const double v = acc[q] * a.map_sc[A.map0 + ia] * a.map_sc[C.map0 + icc];
          a.out[static_cast<int64_t>(fa) * a.n + fc] = v;
          a.out[static_cast<int64_t>(fc) * a.n + fa] = v;
        } else {
          const int fb = a.map_fn[B.map0 + ib];
          if (fa < 0 || fb < 0 || fc < 0 || (sym && ia > ib)) continue;
          const double v = acc[q] * a.map_sc[A.map0 + ia] * a.map_sc[B.map0 + ib] * a.map_sc[C.map0 + icc];
          const int64_t row = static_cast<int64_t>(fc) * a.n * a.n;
          a.out[row + static_cast<int64_t>(fa) * a.n + fb] = v;
          a.out[row + static_cast<int64_t>(fb) * a.n + fa] = v;
        }
      }
    }
  }
}

// Test hook kernel: F_n(T) for every T of a list, as the integral kernels evaluate it (table path).
__global__ void boys_kernel(const double* T, int64_t count, int nmax, const double* tab, double* out) {
  double F[kMaxLSum + 1];
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    boys_table_eval(nmax, T[i], tab, F);
    for (int n = 0; n <= nmax; ++n) out[i * (nmax + 1) + n] = F[n];
  }
}


bool launch_class_any(int la, int lb, int lc, const ClassArgs& a, cudaStream_t s) {
  return launch_class_sp(la, lb, lc, a, s) || launch_class_split(la, lb, lc, a, s) ||
         launch_class_dp01(la, lb, lc, a, s) || launch_class_dp2(la, lb, lc, a, s);
}

double common_factor(int l) {
  if (l == 0) return 1.0 / std::sqrt(4.0 * M_PI);
  if (l == 1) return std::sqrt(3.0 / (4.0 * M_PI));
  return 1.0;
}

// Host shell list built from a flattened basis-function list.
struct HostShells {
  std::vector<DShell> sh;
  std::vector<double> ex, co, sc;
  std::vector<int> fn;
  int lmax = 0;
  int nfirst = 0;  // shells of this list start here in the combined table
};

// Groups the functions into shells: a run of len(components(l)) consecutive functions in libcint's
// component order with equal centre, l and exponents and proportional coefficients is one shell (the
// first function's coefficients, each component scaled by its coefficient ratio); any other function is
// a shell of its own whose other components are not written.
void group_shells(const rr_basis* b, const char* what, HostShells& hs) {
  RR_REQUIRE(b != nullptr && b->n >= 0, RR_ERR_ARG, std::string(what) + ": null basis");
  const int64_t n = b->n;
  if (n == 0) return;
  RR_REQUIRE(b->center && b->lxyz && b->prim_offset && b->exponents && b->coefficients, RR_ERR_ARG,
             std::string(what) + ": null basis array");
  RR_REQUIRE(b->prim_offset[0] == 0, RR_ERR_ARG, std::string(what) + ": prim_offset[0] must be 0");
  for (int64_t i = 0; i < n; ++i) {
    const int l = b->lxyz[3 * i] + b->lxyz[3 * i + 1] + b->lxyz[3 * i + 2];
    RR_REQUIRE(b->lxyz[3 * i] >= 0 && b->lxyz[3 * i + 1] >= 0 && b->lxyz[3 * i + 2] >= 0 && l <= kMaxL, RR_ERR_ARG,
               std::string(what) + ": Cartesian exponents must be >= 0 with l <= 6");
    RR_REQUIRE(b->prim_offset[i + 1] > b->prim_offset[i], RR_ERR_ARG,
               std::string(what) + ": every function needs at least one primitive");
    for (int64_t q = b->prim_offset[i]; q < b->prim_offset[i + 1]; ++q)
      RR_REQUIRE(b->exponents[q] > 0.0 && std::isfinite(b->exponents[q]) && std::isfinite(b->coefficients[q]),
                 RR_ERR_ARG, std::string(what) + ": exponents must be positive and finite");
  }
  auto comp_index = [](int l, int lx, int ly) {
    int idx = 0;
    for (int x = l; x >= 0; --x)
      for (int y = l - x; y >= 0; --y) {
        if (x == lx && y == ly) return idx;
        ++idx;
      }
    return -1;
  };
  int64_t i = 0;
  while (i < n) {
    const int* c0 = b->lxyz + 3 * i;
    const int l = c0[0] + c0[1] + c0[2];
    const int nc = ncart(l);
    const int64_t p0 = b->prim_offset[i], np = b->prim_offset[i + 1] - p0;
    bool ok = i + nc <= n;
    for (int k = 0; ok && k < nc; ++k) {
      const int64_t f = i + k;
      const int* c = b->lxyz + 3 * f;
      ok = c[0] + c[1] + c[2] == l && comp_index(l, c[0], c[1]) == k && b->center[3 * f] == b->center[3 * i] &&
           b->center[3 * f + 1] == b->center[3 * i + 1] && b->center[3 * f + 2] == b->center[3 * i + 2] &&
           b->prim_offset[f + 1] - b->prim_offset[f] == np;
      if (!ok) break;
      const int64_t pf = b->prim_offset[f];
      const double r = b->coefficients[pf] / b->coefficients[p0];
      for (int64_t q = 0; ok && q < np; ++q) {
        ok = b->exponents[pf + q] == b->exponents[p0 + q];
        const double want = b->coefficients[p0 + q] * r;
        ok = ok && std::fabs(b->coefficients[pf + q] - want) <= 1e-13 * std::fabs(want) + 1e-300;
      }
    }
    DShell s;
    s.x = b->center[3 * i];
    s.y = b->center[3 * i + 1];
    s.z = b->center[3 * i + 2];
    s.l = l;
    s.nprim = static_cast<int>(np);
    s.prim0 = static_cast<int>(hs.ex.size());
    s.map0 = static_cast<int>(hs.fn.size());
    const double f = common_factor(l);
    for (int64_t q = 0; q < np; ++q) {
      hs.ex.push_back(b->exponents[p0 + q]);
      hs.co.push_back(b->coefficients[p0 + q] * f);
    }
    hs.fn.resize(hs.fn.size() + nc, -1);
    hs.sc.resize(hs.sc.size() + nc, 0.0);
    if (ok) {
      for (int k = 0; k < nc; ++k) {
        hs.fn[s.map0 + k] = static_cast<int>(i + k);
        hs.sc[s.map0 + k] = b->coefficients[b->prim_offset[i + k]] / b->coefficients[p0];
      }
      i += nc;
    } else {
      const int k = comp_index(l, c0[0], c0[1]);
      hs.fn[s.map0 + k] = static_cast<int>(i);
      hs.sc[s.map0 + k] = 1.0;
      i += 1;
    }
    hs.sh.push_back(s);
    hs.lmax = std::max(hs.lmax, l);
  }
}

// Appends `src` to the combined table `dst` (prim and map offsets shifted).
void append_shells(HostShells& dst, const HostShells& src) {
  const int pe = static_cast<int>(dst.ex.size()), pm = static_cast<int>(dst.fn.size());
  for (DShell s : src.sh) {
    s.prim0 += pe;
    s.map0 += pm;
    dst.sh.push_back(s);
  }
  dst.ex.insert(dst.ex.end(), src.ex.begin(), src.ex.end());
  dst.co.insert(dst.co.end(), src.co.begin(), src.co.end());
  dst.fn.insert(dst.fn.end(), src.fn.begin(), src.fn.end());
  dst.sc.insert(dst.sc.end(), src.sc.begin(), src.sc.end());
  dst.lmax = std::max(dst.lmax, src.lmax);
}

template <typename T>
void upload(DevBuf<T>& d, const std::vector<T>& h, cudaStream_t s) {
  d.alloc(std::max<size_t>(h.size(), 1));
  if (!h.empty()) RR_CUDA(cudaMemcpyAsync(d.p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s));
}

// The Boys table of the current device, built once (kept until exit, 144 KB).
const double* boys_table(cudaStream_t s) {
  static double* tab[kMaxDevices] = {};
  static std::mutex mu;
  const int dev = current_device();
  std::lock_guard<std::mutex> lock(mu);
  if (!tab[dev]) {
    double* t = nullptr;
    RR_CUDA(cudaMalloc(&t, sizeof(double) * kBoysPoints * kBoysOrders));
    boys_table_kernel<<<(kBoysPoints + 127) / 128, 128, 0, s>>>(t);
    RR_LAUNCH_CHECK();
    RR_CUDA(cudaStreamSynchronize(s));
    tab[dev] = t;
  }
  return tab[dev];
}

// Device copy of the combined shell table.
struct DevShells {
  DevBuf<DShell> sh;
  DevBuf<double> ex, co, sc;
  DevBuf<int> fn;
  DevShells(const HostShells& all, cudaStream_t s) {
    upload(sh, all.sh, s);
    upload(ex, all.ex, s);
    upload(co, all.co, s);
    upload(sc, all.sc, s);
    upload(fn, all.fn, s);
  }
};

// Launches eri_kernel (warp per item) over pairs x the ket shells `cidx` (device list of nc).
void launch_eri(const DevShells& d, const int2* pairs, int64_t npairs, const int* cidx, int64_t nc, int la_max,
                int lc_max, bool metric, int64_t n, double* out, const double* boys, cudaStream_t s) {
  if (npairs == 0 || nc == 0) return;
  IntArgs a{};
  a.sh = d.sh.p;
  a.ex = d.ex.p;
  a.co = d.co.p;
  a.map_fn = d.fn.p;
  a.map_sc = d.sc.p;
  a.pairs = pairs;
  a.npairs = npairs;
  a.cidx = cidx;
  a.nc = nc;
  a.metric = metric ? 1 : 0;
  a.n = n;
  a.out = out;
  a.boys = boys;
  a.la_max = la_max;
  a.lab_max = 2 * la_max;
  a.lc_max = lc_max;
  a.L_max = 2 * la_max + lc_max;
  RR_REQUIRE(a.L_max <= kMaxLSum, RR_ERR_ARG, "integrals: la + lb + lc above 18");
  const int esz = (a.la_max + 1) * (a.la_max + 1) * (a.lab_max + 1);
  const int per_warp = 3 * esz + (a.lc_max + 1) * (a.lc_max + 1) + (a.L_max + 1) * (a.L_max + 2) * (a.L_max + 3) / 6 +
                       (a.L_max + 1);
  const size_t smem = sizeof(double) * per_warp * (kIntThreads / 32);
  RR_REQUIRE(smem <= 227 * 1024, RR_ERR_ARG, "integrals: angular momenta too high for the shared-memory tables");
  RR_CUDA(cudaFuncSetAttribute(eri_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  int sms = 0, per_sm = 0;
  const int dev = current_device();
  RR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, eri_kernel, kIntThreads, smem));
  const int64_t items = npairs * nc;
  const int64_t want = (items + kIntThreads / 32 - 1) / (kIntThreads / 32);
  const int grid = static_cast<int>(
      std::max<int64_t>(1, std::min<int64_t>(want, static_cast<int64_t>(sms) * std::max(per_sm, 1) * 4)));
  eri_kernel<<<grid, kIntThreads, smem, s>>>(a);
  RR_LAUNCH_CHECK();
}

struct IntCtx {
  cudaStream_t s = nullptr;
  bool own = false;
  explicit IntCtx(const rr_opts* o) {
    if (o && o->stream) {
      s = static_cast<cudaStream_t>(o->stream);
    } else {
      RR_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      own = true;
    }
  }
  ~IntCtx() {
    if (own && s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
};

void aux_metric_device(const rr_basis* aux, double* M, cudaStream_t s) {
  HostShells hs;
  group_shells(aux, "auxMetric", hs);
  const int na = static_cast<int>(hs.sh.size());
  if (na == 0) return;
  const double* boys = boys_table(s);
  // the constant function 1 as the second bra factor: one primitive of exponent 0, coefficient 1
  // (beta = 0 makes its centre irrelevant: P = A, K = 1)
  HostShells unit;
  unit.sh.push_back(DShell{0.0, 0.0, 0.0, 0, 1, 0, 0});
  unit.ex.push_back(0.0);
  unit.co.push_back(1.0);
  unit.fn.push_back(-1);
  unit.sc.push_back(0.0);
  HostShells all = hs;
  const int iu = static_cast<int>(all.sh.size());
  append_shells(all, unit);
  // bra shells (A, unit) and ket shells, both by angular momentum; a (l_A, 0 | l_C) class kernel in
  // metric mode where one exists (items with C < A skipped there), else the warp kernel
  std::vector<int2> pairs;
  std::vector<int> cidx;
  std::vector<int64_t> p0(kMaxL + 2, 0), c0(kMaxL + 2, 0);
  for (int l = 0; l <= kMaxL; ++l) {
    for (int i = 0; i < na; ++i)
      if (hs.sh[i].l == l) {
        pairs.push_back(make_int2(i, iu));
        cidx.push_back(i);
      }
    p0[l + 1] = static_cast<int64_t>(pairs.size());
    c0[l + 1] = static_cast<int64_t>(cidx.size());
  }
  DevShells d(all, s);
  DevBuf<int2> dp;
  DevBuf<int> dc;
  upload(dp, pairs, s);
  upload(dc, cidx, s);
  ClassArgs ca{d.sh.p, d.ex.p, d.co.p, d.fn.p, d.sc.p, nullptr, 0, nullptr, 0, aux->n, M, boys, 1};
  for (int la = 0; la <= kMaxL; ++la)
    for (int lc = 0; lc <= kMaxL; ++lc) {
      const int64_t np = p0[la + 1] - p0[la], nc = c0[lc + 1] - c0[lc];
      if (np == 0 || nc == 0) continue;
      ca.pairs = dp.p + p0[la];
      ca.npairs = np;
      ca.cidx = dc.p + c0[lc];
      ca.ncs = nc;
      if (!launch_class_any(la, 0, lc, ca, s))
        launch_eri(d, dp.p + p0[la], np, dc.p + c0[lc], nc, hs.lmax, hs.lmax, true, aux->n, M, boys, s);
    }
  RR_CUDA(cudaStreamSynchronize(s));  // the tables are freed on return
}

void three_center_raw_device(const rr_basis* orb, const rr_basis* aux, double* raw, cudaStream_t s) {
  HostShells ho, ha;
  group_shells(orb, "threeCenterIntegralsRaw (orbital basis)", ho);
  group_shells(aux, "threeCenterIntegralsRaw (aux basis)", ha);
  const int no = static_cast<int>(ho.sh.size()), na = static_cast<int>(ha.sh.size());
  if (no == 0 || na == 0) return;
  const double* boys = boys_table(s);
  HostShells all = ho;
  append_shells(all, ha);
  // pairs (i <= j) by class (l_A >= l_B after a swap: both halves of the pq symmetry are written),
  // within a class by primitive count (threads of a warp loop alike); aux shells by l
  std::vector<std::vector<int2>> by_class((kMaxL + 1) * (kMaxL + 1));
  for (int i = 0; i < no; ++i)
    for (int j = i; j < no; ++j) {
      int a = i, b = j;
      if (ho.sh[a].l < ho.sh[b].l) std::swap(a, b);
      by_class[ho.sh[a].l * (kMaxL + 1) + ho.sh[b].l].push_back(make_int2(a, b));
    }
  std::vector<std::vector<int>> aux_by_l(kMaxL + 1);
  for (int c = 0; c < na; ++c) aux_by_l[ha.sh[c].l].push_back(no + c);
  std::vector<int2> pairs;
  std::vector<int> cidx;
  struct Range { int la, lb; int64_t p0, np; };
  std::vector<Range> ranges;
  for (int la = 0; la <= kMaxL; ++la)
    for (int lb = 0; lb <= la; ++lb) {
      auto& v = by_class[la * (kMaxL + 1) + lb];
      if (v.empty()) continue;
      std::stable_sort(v.begin(), v.end(), [&](int2 x, int2 y) {
        return ho.sh[x.x].nprim * ho.sh[x.y].nprim > ho.sh[y.x].nprim * ho.sh[y.y].nprim;
      });
      ranges.push_back(Range{la, lb, static_cast<int64_t>(pairs.size()), static_cast<int64_t>(v.size())});
      pairs.insert(pairs.end(), v.begin(), v.end());
    }
  std::vector<int64_t> c0(kMaxL + 2, 0);
  for (int l = 0; l <= kMaxL; ++l) {
    c0[l + 1] = c0[l] + static_cast<int64_t>(aux_by_l[l].size());
    cidx.insert(cidx.end(), aux_by_l[l].begin(), aux_by_l[l].end());
  }
  DevShells d(all, s);
  DevBuf<int2> dp;
  DevBuf<int> dc;
  upload(dp, pairs, s);
  upload(dc, cidx, s);
  ClassArgs ca{d.sh.p, d.ex.p, d.co.p, d.fn.p, d.sc.p, nullptr, 0, nullptr, 0, orb->n, raw, boys, 0};
  for (const Range& r : ranges)
    for (int lc = 0; lc <= kMaxL; ++lc) {
      const int64_t nc = c0[lc + 1] - c0[lc];
      if (nc == 0) continue;
      ca.pairs = dp.p + r.p0;
      ca.npairs = r.np;
      ca.cidx = dc.p + c0[lc];
      ca.ncs = nc;
      if (!launch_class_any(r.la, r.lb, lc, ca, s))
        launch_eri(d, dp.p + r.p0, r.np, dc.p + c0[lc], nc, ho.lmax, ha.lmax, false, orb->n, raw, boys, s);
    }
  RR_CUDA(cudaStreamSynchronize(s));  // the tables are freed on return
}

template <typename F>
int int_api(F&& f) {
  try {
    set_last_error("");
    f();
    return RR_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return RR_ERR_NOMEM;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return RR_ERR_CUDA;
  }
}

}  // namespace
}  // namespace rr

extern "C" {

int rr_int_aux_metric(const rr_basis* aux, double* metric, const rr_opts* opts) {
  return rr::int_api([&] {
    RR_REQUIRE(aux && metric, RR_ERR_ARG, "auxMetric: null argument");
    RR_REQUIRE(!opts || opts->precision == RR_PREC_FP64, RR_ERR_UNSUPPORTED, "auxMetric: precision");
    rr::IntCtx c(opts);
    const int64_t n = aux->n;
    if (n == 0) return;
    const bool host = !opts || opts->mem == RR_MEM_HOST;
    rr::DevBuf<double> buf;
    double* M = metric;
    if (host) {
      buf.alloc(static_cast<size_t>(n * n));
      M = buf.p;
    }
    rr::aux_metric_device(aux, M, c.s);
    if (host) {
      RR_CUDA(cudaMemcpyAsync(metric, M, sizeof(double) * n * n, cudaMemcpyDeviceToHost, c.s));
      RR_CUDA(cudaStreamSynchronize(c.s));
    }
  });
}

int rr_int_three_center_raw(const rr_basis* basis, const rr_basis* aux, double* raw, const rr_opts* opts) {
  return rr::int_api([&] {
    RR_REQUIRE(basis && aux && raw, RR_ERR_ARG, "threeCenterIntegralsRaw: null argument");
    RR_REQUIRE(!opts || opts->precision == RR_PREC_FP64, RR_ERR_UNSUPPORTED, "threeCenterIntegralsRaw: precision");
    rr::IntCtx c(opts);
    const int64_t n = basis->n, na = aux->n;
    if (n == 0 || na == 0) return;
    const bool host = !opts || opts->mem == RR_MEM_HOST;
    rr::DevBuf<double> buf;
    double* out = raw;
    if (host) {
      buf.alloc(static_cast<size_t>(na * n * n));
      out = buf.p;
    }
    rr::three_center_raw_device(basis, aux, out, c.s);
    if (host) {
      RR_CUDA(cudaMemcpyAsync(raw, out, sizeof(double) * na * n * n, cudaMemcpyDeviceToHost, c.s));
      RR_CUDA(cudaStreamSynchronize(c.s));
    }
  });
}

int rr_ri_create_basis(const rr_basis* basis, const rr_basis* aux, double metric_threshold, const double* t,
                       int64_t n_out, rr_ri_handle* out, int64_t* naux_kept, rr_rank_report* report) {
  return rr::int_api([&] {
    RR_REQUIRE(basis && aux && out, RR_ERR_ARG, "rr_ri_create_basis: null argument");
    *out = nullptr;
    const int64_t n = basis->n, na = aux->n;
    RR_REQUIRE(n >= 1 && na >= 1, RR_ERR_ARG, "rr_ri_create_basis: empty basis");
    rr::IntCtx c(nullptr);
    rr::DevBuf<double> M(static_cast<size_t>(na * na)), X(static_cast<size_t>(na * na)),
        raw(static_cast<size_t>(na * n * n)), td;
    rr::aux_metric_device(aux, M.p, c.s);
    rr_opts dev{};
    dev.mem = RR_MEM_DEVICE;
    dev.precision = RR_PREC_FP64;
    dev.stream = c.s;
    dev.sync = 1;
    int64_t kept = 0;
    rr_rank_report rep{};
    rr::canonical_orthogonalize(M.p, na, false, metric_threshold, X.p, &kept, &rep, &dev);
    rr::three_center_raw_device(basis, aux, raw.p, c.s);
    if (t) {
      RR_REQUIRE(n_out >= 1, RR_ERR_ARG, "rr_ri_create_basis: n_out must be >= 1 with t");
      td.alloc(static_cast<size_t>(n * n_out));
      RR_CUDA(cudaMemcpyAsync(td.p, t, sizeof(double) * n * n_out, cudaMemcpyHostToDevice, c.s));
    }
    RR_CUDA(cudaStreamSynchronize(c.s));
    const int rc = rr_ri_create_raw(raw.p, na, n, X.p, kept, t ? td.p : nullptr, n_out, RR_MEM_DEVICE, out);
    if (rc != RR_OK) throw rr::Error(rc, rr_last_error());
    if (naux_kept) *naux_kept = kept;
    if (report) *report = rep;
  });
}

int rr_test_boys(const double* T, int64_t count, int32_t nmax, double* out) {
  return rr::int_api([&] {
    RR_REQUIRE(T && out && count >= 0 && nmax >= 0 && nmax <= rr::kMaxLSum, RR_ERR_ARG,
               "rr_test_boys: need 0 <= nmax <= 18 and non-null arrays");
    if (count == 0) return;
    rr::DevBuf<double> dT(static_cast<size_t>(count)), dF(static_cast<size_t>(count * (nmax + 1)));
    RR_CUDA(cudaMemcpy(dT.p, T, sizeof(double) * count, cudaMemcpyHostToDevice));
    const double* tab = rr::boys_table(nullptr);
    rr::boys_kernel<<<static_cast<int>(std::min<int64_t>((count + 127) / 128, 1184)), 128>>>(dT.p, count, nmax, tab,
                                                                                          dF.p);
    RR_LAUNCH_CHECK();
    RR_CUDA(cudaMemcpy(out, dF.p, sizeof(double) * count * (nmax + 1), cudaMemcpyDeviceToHost));
  });
}

}  // extern "C"
