// Nonrelativistic half-transform T[P] = Ct B^P (reference: the per-aux-index DGEMM of
// src/NON_REL/NonRelFockMatrixRi.cpp:84-90) on the m16n8k8 FP64 tensor-core shape of sm_90+.
//
// The product is computed transposed, T[P]^T = B^P^T Ct^T: its M is the AO count n (16-row fragments
// cover any n that is a multiple of 16 without padding, unlike the occupied count), N = nocc (8-column
// fragments), K = n.  A CTA owns an 80 x 40 block of T[P]^T (five warps of 16 x 40: one A fragment and five
// B fragments per k8 step) and stores it transposed into T[P] (nocc x n, row-major, the layout the
// exchange SYRK reads).  A 3-stage cp.async ring stages 16-deep k tiles of B^P (rows k, AO columns
// contiguous) and of Ct; the shared-memory pitches are 4 (mod 16) doubles, so the fragment loads of a
// half-warp touch 16 distinct 8-byte bank pairs.
#include <algorithm>
#include <cstdlib>
#include <string>

#include "gemm_f64.cuh"

namespace rr {
namespace {

constexpr int HT_BM = 80, HT_BN = 40, HT_KT = 16, HT_STAGES = 3, HT_THREADS = 160;
constexpr int HT_LDA = HT_BM + 4;  // sA[k][m]: 84 = 4 (mod 16), even (16-byte cp.async destinations)
constexpr int HT_LDB = HT_KT + 4;  // sB[n][k]: 20 = 4 (mod 16)
constexpr int HT_SA = HT_KT * HT_LDA, HT_SB = HT_BN * HT_LDB, HT_STAGE = HT_SA + HT_SB;
constexpr int HT_SMEM = HT_STAGES * HT_STAGE * 8;

__device__ __forceinline__ void cp16(uint32_t saddr, const void* g, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(g), "r"(bytes));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// D(16x8) += A(16x8, row) B(8x8, col), FP64.  Fragments (g = lane / 4, t = lane % 4):
// a0 = A[g][t], a1 = A[g+8][t], a2 = A[g][t+4], a3 = A[g+8][t+4]; b0 = B[t][g], b1 = B[t+4][g];
// c0 = D[g][2t], c1 = D[g][2t+1], c2 = D[g+8][2t], c3 = D[g+8][2t+1].
__device__ __forceinline__ void dmma16(double (&c)[4], double a0, double a1, double a2, double a3, double b0, double b1) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
               : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
               : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

struct HtArgs {
  const double* Ct;  // nocc x n, row pitch n
  const double* B;   // naux rows of pitch doubles (n x n each)
  double* T;         // naux x nocc x n
  int64_t n, nocc, pitch, p0;
};

__global__ void __launch_bounds__(HT_THREADS) ht_dmma16_kernel(const HtArgs a) {
  extern __shared__ __align__(16) double smem[];
  const int64_t j0 = static_cast<int64_t>(blockIdx.x) * HT_BM;  // AO columns of B^P (rows of T^T)
  const int64_t i0 = static_cast<int64_t>(blockIdx.y) * HT_BN;  // occupied rows of T
  const int64_t P = a.p0 + blockIdx.z;
  const double* Bp = a.B + P * a.pitch;
  const int64_t n = a.n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  const int ktiles = static_cast<int>((n + HT_KT - 1) / HT_KT);

  auto load = [&](int stage, int kt) {
    const int64_t k0 = static_cast<int64_t>(kt) * HT_KT;
    const uint32_t sa = sbase + static_cast<uint32_t>(stage * HT_STAGE * 8);
    const uint32_t sb = sa + HT_SA * 8;
    // B^P rows k0..k0+15, AO columns j0..j0+79: 640 16-byte chunks (two doubles each)
#pragma unroll
    for (int e = tid; e < HT_KT * HT_BM / 2; e += HT_THREADS) {
      const int r = e / (HT_BM / 2), c = 2 * (e % (HT_BM / 2));
      const int64_t k = k0 + r, j = j0 + c;
      const int nvalid = k < n ? static_cast<int>(max(int64_t(0), min(int64_t(2), n - j))) : 0;
      cp16(sa + static_cast<uint32_t>((r * HT_LDA + c) * 8), nvalid ? Bp + k * n + j : Bp, nvalid * 8);
    }
    // Ct rows i0..i0+39, columns k0..k0+15: 320 chunks
#pragma unroll
    for (int e = tid; e < HT_BN * HT_KT / 2; e += HT_THREADS) {
      const int r = e / (HT_KT / 2), c = 2 * (e % (HT_KT / 2));
      const int64_t i = i0 + r, k = k0 + c;
      const int nvalid = i < a.nocc ? static_cast<int>(max(int64_t(0), min(int64_t(2), n - k))) : 0;
      cp16(sb + static_cast<uint32_t>((r * HT_LDB + c) * 8), nvalid ? a.Ct + i * n + k : a.Ct, nvalid * 8);
    }
  };

  double acc[5][4];
#pragma unroll
  for (int jb = 0; jb < 5; ++jb)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[jb][q] = 0.0;

#pragma unroll
  for (int s = 0; s < HT_STAGES - 1; ++s) {
    if (s < ktiles) load(s, s);
    cp_commit();
  }
  const int m = warp * 16 + g;  // this lane's A rows m and m + 8 within the tile
  for (int kt = 0; kt < ktiles; ++kt) {
    cp_wait<HT_STAGES - 2>();
    __syncthreads();
    const double* sA = smem + (kt % HT_STAGES) * HT_STAGE;
    const double* sB = sA + HT_SA;
#pragma unroll
    for (int ks = 0; ks < HT_KT / 8; ++ks) {
      const int k = ks * 8 + t;
      const double a0 = sA[k * HT_LDA + m], a1 = sA[k * HT_LDA + m + 8];
      const double a2 = sA[(k + 4) * HT_LDA + m], a3 = sA[(k + 4) * HT_LDA + m + 8];
#pragma unroll
      for (int jb = 0; jb < 5; ++jb) {
        const double b0 = sB[(jb * 8 + g) * HT_LDB + k], b1 = sB[(jb * 8 + g) * HT_LDB + k + 4];
        dmma16(acc[jb], a0, a1, a2, a3, b0, b1);
      }
    }
    const int nk = kt + HT_STAGES - 1;
    if (nk < ktiles) load(nk % HT_STAGES, nk);
    cp_commit();
  }
  cp_wait<0>();
  // D = T^T block: D[row = AO j][col = occupied i]; stored into T[P][i][j]
  double* Tp = a.T + P * a.nocc * n;
#pragma unroll
  for (int jb = 0; jb < 5; ++jb)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int64_t j = j0 + warp * 16 + g + (q >= 2 ? 8 : 0);
      const int64_t i = i0 + jb * 8 + 2 * t + (q & 1);
      if (j < n && i < a.nocc) Tp[i * n + j] = acc[jb][q];
    }
}

}  // namespace

bool half_transform_m16(const double* Ct, int64_t nocc, const double* B, int64_t pitch, int64_t naux, int64_t n,
                        double* T, cudaStream_t s) {
  // 16-byte cp.async sources: even n and pitch, 16-byte aligned bases
  auto al = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
  if (n % 2 != 0 || pitch % 2 != 0 || !al(Ct) || !al(B) || nocc <= 0 || n <= 0) return false;
  static std::atomic<bool> attr[kMaxDevices];
  once_per_device(attr, [] {
    RR_CUDA(cudaFuncSetAttribute(ht_dmma16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, HT_SMEM));
    RR_CUDA(cudaFuncSetAttribute(ht_dmma16_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
  });
  for (int64_t p0 = 0; p0 < naux; p0 += 65535) {
    const int64_t cnt = std::min<int64_t>(65535, naux - p0);
    HtArgs a{Ct, B, T, n, nocc, pitch, p0};
    dim3 grid(static_cast<unsigned>((n + HT_BM - 1) / HT_BM), static_cast<unsigned>((nocc + HT_BN - 1) / HT_BN),
              static_cast<unsigned>(cnt));
    ht_dmma16_kernel<<<grid, HT_THREADS, HT_SMEM, s>>>(a);
    RR_LAUNCH_CHECK();
  }
  return true;
}

int half_transform_kind() {
  static const int kind = [] {
    const char* e = std::getenv("RR_HALF_TRANSFORM");
    if (e && std::string(e) == "m8") return 0;
    if (e && std::string(e) == "m16") return 1;
    return 1;  // 1.633 against 1.656 ms per n = 400, naux = 1600, nocc = 40 build (50 builds each)
  }();
  return kind;
}

}  // namespace rr
