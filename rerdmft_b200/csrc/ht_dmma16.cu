// Nonrelativistic half-transform T[P] = Ct B^P (reference: the per-aux-index DGEMM of
// src/NON_REL/NonRelFockMatrixRi.cpp:84-90) on the m16n8k8 FP64 tensor-core shape of sm_90+.
//
// The product is computed transposed, T[P]^T = B^P^T Ct^T: its M is the AO count n (16-row fragments
// cover any n that is a multiple of 16 without padding, unlike the occupied count), N = nocc (8-column
// fragments), K = n.  Each warp owns a 16 x 40 block of T[P]^T (one A fragment and five B fragments per
// k8 step) and stores it transposed into T[P] (nocc x n, row-major, the layout the exchange SYRK reads).
// The default CTA is two such warps (32 AO columns) over a 3-stage cp.async ring of 16-deep k tiles of
// B^P (rows k, AO columns contiguous) and of Ct.  Timed alone at n = 400, naux = 1600, nocc = 40 a
// 5-stage ring is the fastest tiling (0.723 ms against 0.824 ms for five warps over 3 stages and
// 0.76-1.19 ms for the others kept for measurement, half_transform_m16's config, the warp-specialised
// bulk-copy pipeline included); inside the Fock build, where the exchange overlaps the Coulomb passes on
// another stream, the 3-stage ring (27 KB of shared memory a CTA against 45 KB) gave 1.565 ms a build
// against 1.636 ms for the 5-stage one and 1.615-1.619 ms for (4,16,4) and (2,16,4).
#include <algorithm>
#include <cstdlib>
#include <string>

#include "gemm_f64.cuh"
#include "tma_util.cuh"

namespace rr {
namespace {

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

// WARPS warps per CTA, each a 16-row slice of the CTA's BM = 16 WARPS AO columns times 40 occupied
// rows; KT-deep k tiles in a STAGES-deep ring.  Shared-memory pitches are 4 (mod 16) doubles, so the
// fragment loads of a half-warp touch 16 distinct 8-byte bank pairs.
template <int WARPS, int KT, int STAGES>
struct HtCfg {
  static constexpr int BM = 16 * WARPS, BN = 40, THREADS = 32 * WARPS;
  static constexpr int LDA = BM + 4;  // sA[k][m]
  static constexpr int LDB = KT + 4;  // sB[n][k]
  static constexpr int SA = KT * LDA, SB = BN * LDB, STAGE = SA + SB;
  static constexpr int SMEM = STAGES * STAGE * 8;
  static_assert(LDA % 16 == 4 && LDB % 16 == 4, "pitches must be 4 (mod 16)");
};

template <int WARPS, int KT, int STAGES>
__global__ void __launch_bounds__(32 * WARPS) ht_dmma16_kernel(const HtArgs a) {
  using CF = HtCfg<WARPS, KT, STAGES>;
  constexpr int BM = CF::BM, BN = CF::BN, THREADS = CF::THREADS, LDA = CF::LDA, LDB = CF::LDB;
  extern __shared__ __align__(16) double smem[];
  const int64_t j0 = static_cast<int64_t>(blockIdx.x) * BM;  // AO columns of B^P (rows of T^T)
  const int64_t i0 = static_cast<int64_t>(blockIdx.y) * BN;  // occupied rows of T
  const int64_t P = a.p0 + blockIdx.z;
  const double* Bp = a.B + P * a.pitch;
  const int64_t n = a.n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  const int ktiles = static_cast<int>((n + KT - 1) / KT);

  auto load = [&](int stage, int kt) {
    const int64_t k0 = static_cast<int64_t>(kt) * KT;
    const uint32_t sa = sbase + static_cast<uint32_t>(stage * CF::STAGE * 8);
    const uint32_t sb = sa + CF::SA * 8;
    // B^P rows k0 .. k0+KT-1, AO columns j0 .. j0+BM-1 (16-byte chunks of two doubles)
#pragma unroll
    for (int e = tid; e < KT * BM / 2; e += THREADS) {
      const int r = e / (BM / 2), c = 2 * (e % (BM / 2));
      const int64_t k = k0 + r, j = j0 + c;
      const int nvalid = k < n ? static_cast<int>(max(int64_t(0), min(int64_t(2), n - j))) : 0;
      cp16(sa + static_cast<uint32_t>((r * LDA + c) * 8), nvalid ? Bp + k * n + j : Bp, nvalid * 8);
    }
    // Ct rows i0 .. i0+39, columns k0 .. k0+KT-1
#pragma unroll
    for (int e = tid; e < BN * KT / 2; e += THREADS) {
      const int r = e / (KT / 2), c = 2 * (e % (KT / 2));
      const int64_t i = i0 + r, k = k0 + c;
      const int nvalid = i < a.nocc ? static_cast<int>(max(int64_t(0), min(int64_t(2), n - k))) : 0;
      cp16(sb + static_cast<uint32_t>((r * LDB + c) * 8), nvalid ? a.Ct + i * n + k : a.Ct, nvalid * 8);
    }
  };

  double acc[5][4];
#pragma unroll
  for (int jb = 0; jb < 5; ++jb)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[jb][q] = 0.0;

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < ktiles) load(s, s);
    cp_commit();
  }
  const int m = warp * 16 + g;  // this lane's A rows m and m + 8 within the tile
  for (int kt = 0; kt < ktiles; ++kt) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    const double* sA = smem + (kt % STAGES) * CF::STAGE;
    const double* sB = sA + CF::SA;
#pragma unroll
    for (int ks = 0; ks < KT / 8; ++ks) {
      const int k = ks * 8 + t;
      const double a0 = sA[k * LDA + m], a1 = sA[k * LDA + m + 8];
      const double a2 = sA[(k + 4) * LDA + m], a3 = sA[(k + 4) * LDA + m + 8];
#pragma unroll
      for (int jb = 0; jb < 5; ++jb) {
        const double b0 = sB[(jb * 8 + g) * LDB + k], b1 = sB[(jb * 8 + g) * LDB + k + 4];
        dmma16(acc[jb], a0, a1, a2, a3, b0, b1);
      }
    }
    const int nk = kt + STAGES - 1;
    if (nk < ktiles) load(nk % STAGES, nk);
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

// Warp-specialised variant: the five compute warps of the default tiling plus one copy warp that fills
// a STAGES-deep ring with 1-D bulk copies (one per B^P row segment of the tile and one per Ct row
// segment, each into its padded shared-memory row), completing on the stage's `full` mbarrier; the
// compute warps release a stage through its `empty` mbarrier.  No CTA-wide barrier in the main loop,
// so a warp waits only for its data.  Every wait is bounded (status word, then the CTA drains).
template <int STAGES>
__global__ void __launch_bounds__(192, 1) ht_tma16_kernel(const HtArgs a, int* status) {
  using CF = HtCfg<5, 16, STAGES>;
  constexpr int BM = CF::BM, BN = CF::BN, KT = 16, LDA = CF::LDA, LDB = CF::LDB;
  extern __shared__ __align__(16) double smem[];
  __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES];
  const int64_t j0 = static_cast<int64_t>(blockIdx.x) * BM;
  const int64_t i0 = static_cast<int64_t>(blockIdx.y) * BN;
  const int64_t P = a.p0 + blockIdx.z;
  const double* Bp = a.B + P * a.pitch;
  const int64_t n = a.n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ktiles = static_cast<int>((n + KT - 1) / KT);
  if (tid == 0) {
    for (int st = 0; st < STAGES; ++st) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], 5);
    }
    fence_barrier_init();
  }
  __syncthreads();
  bool dead = false;
  // bounded wait: on expiry the status word records 0x10 and this thread skips every later wait
  auto wait = [&](uint64_t* bar, uint32_t parity) -> bool {
    if (dead) return false;
    for (uint32_t i = 0; i < kSpinLimit; ++i)
      if (mbar_try_wait(bar, parity)) return true;
    atomicOr(status, 0x10);
    dead = true;
    return false;
  };
  if (warp == 5) {
    // copy warp
    const int rowsB = static_cast<int>(min(static_cast<int64_t>(BN), a.nocc - i0));
    const uint32_t bytesA = static_cast<uint32_t>(min(static_cast<int64_t>(BM), n - j0) * 8);
    for (int kt = 0; kt < ktiles && !dead; ++kt) {
      const int st = kt % STAGES;
      if (kt >= STAGES) {
        bool ok = true;
        if (lane == 0) ok = wait(&empty[st], ((kt / STAGES) - 1) & 1);
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        if (!ok) { dead = true; break; }
      }
      __syncwarp();
      double* sA = smem + st * CF::STAGE;
      double* sB = sA + CF::SA;
      const int64_t k0 = static_cast<int64_t>(kt) * KT;
      const int rowsA = static_cast<int>(min(static_cast<int64_t>(KT), n - k0));
      const uint32_t bytesB = static_cast<uint32_t>(rowsA * 8);
      // k rows past n (last tile): zeros in both operands
      if (rowsA < KT) {
        for (int e = lane; e < (KT - rowsA) * BM; e += 32) sA[(rowsA + e / BM) * LDA + e % BM] = 0.0;
        for (int e = lane; e < BN * (KT - rowsA); e += 32) sB[(e / (KT - rowsA)) * LDB + rowsA + e % (KT - rowsA)] = 0.0;
      }
      __syncwarp();
      if (lane == 0) mbar_arrive_expect_tx(&full[st], rowsA * bytesA + rowsB * bytesB);
      __syncwarp();
      for (int c = lane; c < rowsA + rowsB; c += 32) {
        if (c < rowsA) tma_load_1d(sA + c * LDA, Bp + (k0 + c) * n + j0, bytesA, &full[st]);
        else tma_load_1d(sB + (c - rowsA) * LDB, a.Ct + (i0 + c - rowsA) * n + k0, bytesB, &full[st]);
      }
    }
    // drain: the copies of the last stages have landed before the CTA may exit
    if (lane == 0) {
      dead = false;
      for (int kt = max(0, ktiles - STAGES); kt < ktiles; ++kt) wait(&full[kt % STAGES], (kt / STAGES) & 1);
    }
    return;
  }
  const int g = lane >> 2, t = lane & 3;
  double acc[5][4];
#pragma unroll
  for (int jb = 0; jb < 5; ++jb)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[jb][q] = 0.0;
  const int m = warp * 16 + g;
  for (int kt = 0; kt < ktiles; ++kt) {
    const int st = kt % STAGES;
    if (!wait(&full[st], (kt / STAGES) & 1)) break;
    const double* sA = smem + st * CF::STAGE;
    const double* sB = sA + CF::SA;
#pragma unroll
    for (int ks = 0; ks < KT / 8; ++ks) {
      const int k = ks * 8 + t;
      const double a0 = sA[k * LDA + m], a1 = sA[k * LDA + m + 8];
      const double a2 = sA[(k + 4) * LDA + m], a3 = sA[(k + 4) * LDA + m + 8];
#pragma unroll
      for (int jb = 0; jb < 5; ++jb) {
        const double b0 = sB[(jb * 8 + g) * LDB + k], b1 = sB[(jb * 8 + g) * LDB + k + 4];
        dmma16(acc[jb], a0, a1, a2, a3, b0, b1);
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[st]);
  }
  if (dead) return;
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

template <int STAGES>
void launch_ht_tma(const HtArgs& base, int64_t naux, int* status, cudaStream_t s) {
  using CF = HtCfg<5, 16, STAGES>;
  auto kern = ht_tma16_kernel<STAGES>;
  static std::atomic<bool> attr[kMaxDevices];
  once_per_device(attr, [&] {
    RR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, CF::SMEM));
    RR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
  });
  for (int64_t p0 = 0; p0 < naux; p0 += 65535) {
    const int64_t cnt = std::min<int64_t>(65535, naux - p0);
    HtArgs a = base;
    a.p0 = p0;
    dim3 grid(static_cast<unsigned>((a.n + CF::BM - 1) / CF::BM), static_cast<unsigned>((a.nocc + CF::BN - 1) / CF::BN),
              static_cast<unsigned>(cnt));
    kern<<<grid, 192, CF::SMEM, s>>>(a, status);
    RR_LAUNCH_CHECK();
  }
}

template <int WARPS, int KT, int STAGES>
void launch_ht(const HtArgs& base, int64_t naux, cudaStream_t s) {
  using CF = HtCfg<WARPS, KT, STAGES>;
  auto kern = ht_dmma16_kernel<WARPS, KT, STAGES>;
  static std::atomic<bool> attr[kMaxDevices];
  once_per_device(attr, [&] {
    RR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, CF::SMEM));
    RR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
  });
  for (int64_t p0 = 0; p0 < naux; p0 += 65535) {
    const int64_t cnt = std::min<int64_t>(65535, naux - p0);
    HtArgs a = base;
    a.p0 = p0;
    dim3 grid(static_cast<unsigned>((a.n + CF::BM - 1) / CF::BM), static_cast<unsigned>((a.nocc + CF::BN - 1) / CF::BN),
              static_cast<unsigned>(cnt));
    kern<<<grid, CF::THREADS, CF::SMEM, s>>>(a);
    RR_LAUNCH_CHECK();
  }
}

}  // namespace

bool half_transform_m16(const double* Ct, int64_t nocc, const double* B, int64_t pitch, int64_t naux, int64_t n,
                        double* T, cudaStream_t s, int config, int* status) {
  // 16-byte cp.async sources: even n and pitch, 16-byte aligned bases
  auto al = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
  if (n % 2 != 0 || pitch % 2 != 0 || !al(Ct) || !al(B) || nocc <= 0 || n <= 0) return false;
  HtArgs a{Ct, B, T, n, nocc, pitch, 0};
  switch (config) {
    case 1: launch_ht<1, 16, 4>(a, naux, s); break;
    case 2: launch_ht<2, 16, 4>(a, naux, s); break;
    case 3: launch_ht<5, 32, 2>(a, naux, s); break;
    case 4: launch_ht<4, 16, 3>(a, naux, s); break;
    case 5: launch_ht<1, 32, 3>(a, naux, s); break;
    case 6: launch_ht<2, 32, 3>(a, naux, s); break;
    case 7:
      if (!status) return false;
      launch_ht_tma<4>(a, naux, status, s);
      break;
    case 8:
      if (!status) return false;
      launch_ht_tma<3>(a, naux, status, s);
      break;
    case 9: launch_ht<2, 16, 5>(a, naux, s); break;
    case 10: launch_ht<5, 16, 3>(a, naux, s); break;
    case 11: launch_ht<2, 16, 6>(a, naux, s); break;
    case 12: launch_ht<4, 16, 4>(a, naux, s); break;
    case 13: launch_ht<3, 16, 4>(a, naux, s); break;
    default: launch_ht<2, 16, 3>(a, naux, s); break;
  }
  return true;
}

int half_transform_kind() {
  static const int kind = [] {
    const char* e = std::getenv("RR_HALF_TRANSFORM");
    if (e && std::string(e) == "m8") return 0;
    return 1;  // m16 (1.565 ms per headline build against 1.656 ms for m8)
  }();
  return kind;
}

int half_transform_config() {
  static const int cfg = [] {
    const char* e = std::getenv("RR_HALF_TRANSFORM");
    if (!e) return 0;
    const std::string v(e);
    if (v.rfind("m16:", 0) != 0) return 0;
    const int c = std::atoi(v.c_str() + 4);
    return c >= 0 && c <= 13 && c != 7 && c != 8 ? c : 0;  // 7 and 8 need a status word
  }();
  return cfg;
}

}  // namespace rr
