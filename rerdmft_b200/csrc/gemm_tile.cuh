// Tile body of the FP64 DMMA GEMM (mma.sync m8n8k4 .f64) shared by the one-problem kernel
// (gemm_f64.cu) and the grouped persistent kernel (gemm_grouped.cu): a 3-stage cp.async pipeline of
// 16-deep k tiles, warp tiles of (MT*8) x (NT*8), optional complex (4M) accumulation, split-K
// partials or the alpha/beta epilogue.
#pragma once

#include "gemm_f64.cuh"

namespace rr {
namespace gk {

constexpr int KT = 16;
constexpr int STAGES = 3;

struct Params {
  int64_t M, N, K;
  const double* A;
  int64_t lda, strideA;
  const double* B;
  int64_t ldb, strideB;
  double* C;
  int64_t ldc, strideC;
  double alpha, beta;
  int64_t batch;
  int splits;
  int64_t kchunk;
  double* work;
  double signA, signB;  // -1 conjugates the imaginary plane of A / B
  int64_t c_plane_rows, c_plane_stride;
  int64_t ccs;  // output column stride
  int upper_only;
  int mirror;  // split-K reduce of an upper-only product also writes the strict lower triangle (+1 / -1; 2: not)
  const double* eE;
  int64_t eld;
  double escale;
  double* eout;
};

__device__ __forceinline__ void cp_async8(uint32_t saddr, const void* g, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(g), "r"(bytes));
}
__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* g, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(g), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// Row pitch (doubles) of the [k][m] / [k][n] tiles: a fragment load reads element (k = t, m = g)
// for lane 4g + t, so with pitch = 4 (mod 16) every half-warp touches 16 distinct 8-byte bank pairs
// (t * pitch + g covers 0..15); an even pitch keeps the 16-byte cp.async destinations aligned.
__host__ __device__ constexpr int pad_mn(int x) { return x + ((4 - x % 16) + 16) % 16; }

template <int MT, int NT, int WM, int WN, bool AK, bool BKM, bool CPLX>
struct Cfg {
  static constexpr int BM = MT * 8 * WM, BN = NT * 8 * WN, THREADS = 32 * WM * WN, PL = CPLX ? 2 : 1;
  static constexpr int A_LD = AK ? (KT + 4) : pad_mn(BM);
  static constexpr int A_SZ = AK ? BM * A_LD : KT * A_LD;
  static constexpr int B_LD = BKM ? (KT + 4) : pad_mn(BN);
  static constexpr int B_SZ = BKM ? BN * B_LD : KT * B_LD;
  static constexpr int STAGE = PL * (A_SZ + B_SZ);
  static constexpr int SMEM_BYTES = STAGES * STAGE * 8;
};

// A tile: AK (A stored M x K, k contiguous) -> smem [BM][A_LD]; else (stored K x M) -> [KT][A_LD].
// B tile: BKM (B stored N x K) -> smem [BN][B_LD]; else (stored K x N) -> [KT][B_LD].
// One output tile (rows m0.., columns n0.., batch x split index bz) of the product p, by the CTA that
// calls it (all its threads); smem: the CTA's dynamic shared memory (Cfg::SMEM_BYTES); eslot: where
// the epilogue dot of this tile goes (EDOT only).  The caller skips the tiles below the diagonal of
// upper-only products.
template <int MT, int NT, int WM, int WN, bool AK, bool BKM, bool CPLX, int V, bool EDOT>
__device__ __forceinline__ void dgemm_tile(const Params& p, int64_t n0, int64_t m0, int64_t bz, double* smem,
                                           int64_t eslot) {
  using CF = Cfg<MT, NT, WM, WN, AK, BKM, CPLX>;
  constexpr int BM = CF::BM, BN = CF::BN, THREADS = CF::THREADS, PL = CF::PL;
  const int64_t b = bz / p.splits;
  const int split = static_cast<int>(bz % p.splits);
  const int64_t kbeg = split * p.kchunk;
  const int64_t kend = min(p.K, kbeg + p.kchunk);
  const int ktiles = kend > kbeg ? static_cast<int>((kend - kbeg + KT - 1) / KT) : 0;

  const double* Ab = p.A + b * p.strideA * PL;
  const double* Bb = p.B + b * p.strideB * PL;
  const int tid = threadIdx.x;
  const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(smem));

  // V = 2: 16-byte copies of two consecutive elements along the contiguous dimension (the host
  // only selects it when every row start and the bases are 16-byte aligned and the contiguous
  // extents are even); V = 1: 8-byte copies.  Out-of-range elements are zero-filled.
  auto load_stage = [&](int stage, int kt) {
    const int64_t k0 = kbeg + static_cast<int64_t>(kt) * KT;
    double* sA = smem + stage * CF::STAGE;
    double* sB = sA + PL * CF::A_SZ;
    constexpr int AW = AK ? KT : BM;  // contiguous width of the A tile
    constexpr int BW = BKM ? KT : BN;
#pragma unroll 4
    for (int e = tid * V; e < BM * KT; e += THREADS * V) {
      const int r = e / AW, c = e % AW;
      int64_t gm, gk;
      if constexpr (AK) { gm = m0 + r; gk = k0 + c; }
      else { gk = k0 + r; gm = m0 + c; }
      const int64_t goff = AK ? gm * p.lda + gk : gk * p.lda + gm;
#pragma unroll
      for (int pl = 0; pl < PL; ++pl) {
        const uint32_t sa = sbase + static_cast<uint32_t>(((sA - smem) + pl * CF::A_SZ + r * CF::A_LD + c) * 8);
        if constexpr (V == 2 && !CPLX) {
          // both elements valid, only the first, or none (contiguous extent even => pairs never straddle)
          const bool row_ok = AK ? gm < p.M : gk < kend;
          const int64_t cpos = AK ? gk : gm;
          const int64_t cend = AK ? kend : p.M;
          const int nvalid = row_ok ? static_cast<int>(max(int64_t(0), min(int64_t(2), cend - cpos))) : 0;
          cp_async16(sa, nvalid ? Ab + goff : Ab, nvalid * 8);
        } else {
          const bool ok = gm < p.M && gk < kend;
          cp_async8(sa, Ab + (ok ? goff : 0) * PL + pl, ok ? 8 : 0);
        }
      }
    }
#pragma unroll 4
    for (int e = tid * V; e < BN * KT; e += THREADS * V) {
      const int r = e / BW, c = e % BW;
      int64_t gn, gk;
      if constexpr (BKM) { gn = n0 + r; gk = k0 + c; }
      else { gk = k0 + r; gn = n0 + c; }
      const int64_t goff = BKM ? gn * p.ldb + gk : gk * p.ldb + gn;
#pragma unroll
      for (int pl = 0; pl < PL; ++pl) {
        const uint32_t sa = sbase + static_cast<uint32_t>(((sB - smem) + pl * CF::B_SZ + r * CF::B_LD + c) * 8);
        if constexpr (V == 2 && !CPLX) {
          const bool row_ok = BKM ? gn < p.N : gk < kend;
          const int64_t cpos = BKM ? gk : gn;
          const int64_t cend = BKM ? kend : p.N;
          const int nvalid = row_ok ? static_cast<int>(max(int64_t(0), min(int64_t(2), cend - cpos))) : 0;
          cp_async16(sa, nvalid ? Bb + goff : Bb, nvalid * 8);
        } else {
          const bool ok = gn < p.N && gk < kend;
          cp_async8(sa, Bb + (ok ? goff : 0) * PL + pl, ok ? 8 : 0);
        }
      }
    }
  };

  const int lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp / WN, wn = warp % WN;
  double acc[MT][NT][PL][2];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int q = 0; q < PL; ++q) acc[i][j][q][0] = acc[i][j][q][1] = 0.0;

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < ktiles) load_stage(s, s);
    cp_async_commit();
  }

  for (int kt = 0; kt < ktiles; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const double* sA = smem + (kt % STAGES) * CF::STAGE;
    const double* sB = sA + PL * CF::A_SZ;
#pragma unroll
    for (int ks = 0; ks < KT / 4; ++ks) {
      const int k = ks * 4 + t;
      double ar[MT], br[NT], ai[MT], bi[NT];
#pragma unroll
      for (int i = 0; i < MT; ++i) {
        const int m = wm * MT * 8 + i * 8 + g;
        const int idx = AK ? m * CF::A_LD + k : k * CF::A_LD + m;
        ar[i] = sA[idx];
        if constexpr (CPLX) ai[i] = p.signA * sA[CF::A_SZ + idx];
      }
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const int n = wn * NT * 8 + j * 8 + g;
        const int idx = BKM ? n * CF::B_LD + k : k * CF::B_LD + n;
        br[j] = sB[idx];
        if constexpr (CPLX) bi[j] = p.signB * sB[CF::B_SZ + idx];
      }
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          dmma(acc[i][j][0][0], acc[i][j][0][1], ar[i], br[j]);
          if constexpr (CPLX) {
            dmma(acc[i][j][0][0], acc[i][j][0][1], -ai[i], bi[j]);
            dmma(acc[i][j][1][0], acc[i][j][1][1], ar[i], bi[j]);
            dmma(acc[i][j][1][0], acc[i][j][1][1], ai[i], br[j]);
          }
        }
    }
    const int nk = kt + STAGES - 1;
    if (nk < ktiles) load_stage(nk % STAGES, nk);
    cp_async_commit();
  }
  cp_async_wait<0>();

  double edot = 0.0;
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int64_t row = m0 + wm * MT * 8 + i * 8 + g;
        const int64_t col = n0 + wn * NT * 8 + j * 8 + 2 * t + e;
        if (row >= p.M || col >= p.N) continue;
        if constexpr (EDOT) edot = fma(p.alpha * acc[i][j][0][e], __ldg(p.eE + row * p.eld + col), edot);
        if (p.splits > 1) {
          double* w = p.work + ((bz * p.M + row) * p.N + col) * PL;
#pragma unroll
          for (int q = 0; q < PL; ++q) w[q] = acc[i][j][q][e];
        } else {
          int64_t rr = row, base = 0;
          if (p.c_plane_rows > 0) { base = (row / p.c_plane_rows) * p.c_plane_stride; rr = row % p.c_plane_rows; }
          double* c = p.C + (base + b * p.strideC + rr * p.ldc + col * p.ccs) * PL;
#pragma unroll
          for (int q = 0; q < PL; ++q) {
            const double v = p.alpha * acc[i][j][q][e];
            c[q] = p.beta != 0.0 ? v + p.beta * c[q] : v;
          }
        }
      }
  if constexpr (EDOT) {
    __syncthreads();  // main loop done with the shared ring: reuse it for the reduction
    for (int o = 16; o > 0; o >>= 1) edot += __shfl_xor_sync(0xffffffffu, edot, o);
    if (lane == 0) smem[warp] = edot;
    __syncthreads();
    if (tid == 0) {
      double tsum = 0.0;
      for (int w = 0; w < THREADS / 32; ++w) tsum += smem[w];
      p.eout[eslot] = p.escale * tsum;
    }
  }
}


// Element idx (< batch M N) of the fixed-order split-K reduction C = alpha * sum_s work[b, s] + beta * C.
template <int PL>
__device__ __forceinline__ void splitk_reduce_elem(const Params& p, int64_t idx) {
  const int64_t b = idx / (p.M * p.N);
  const int64_t rc = idx % (p.M * p.N);
  const int64_t row = rc / p.N, col = rc % p.N;
  if (p.upper_only && row > col) return;  // written as the mirror of (col, row)
  double s[PL];
#pragma unroll
  for (int q = 0; q < PL; ++q) s[q] = 0.0;
  for (int sp = 0; sp < p.splits; ++sp) {
    const double* w = p.work + (((b * p.splits + sp) * p.M + row) * p.N + col) * PL;
#pragma unroll
    for (int q = 0; q < PL; ++q) s[q] += w[q];
  }
  int64_t rr = row, base = 0;
  if (p.c_plane_rows > 0) { base = (row / p.c_plane_rows) * p.c_plane_stride; rr = row % p.c_plane_rows; }
  double* c = p.C + (base + b * p.strideC + rr * p.ldc + col * p.ccs) * PL;
  double v[PL];
#pragma unroll
  for (int q = 0; q < PL; ++q) {
    v[q] = p.alpha * s[q];
    if (p.beta != 0.0) v[q] += p.beta * c[q];
    c[q] = v[q];
  }
  if (p.upper_only && row < col && p.mirror != 2) {
    // the strict lower triangle from the final upper value (mirror requires no plane split and a
    // unit column stride; the lower triangle is never read as beta input here)
    double* t = p.C + (b * p.strideC + col * p.ldc + row) * PL;
    t[0] = p.mirror > 0 ? v[0] : -v[0];
    if (PL == 2) t[1] = p.mirror > 0 ? -v[PL - 1] : v[PL - 1];
  }
}

// Element idx (< batch n n) of the strict lower triangle from the upper one (+1 symmetric /
// Hermitian, -1 antisymmetric).
template <int PL>
__device__ __forceinline__ void mirror_elem(double* C, int64_t n, int64_t ldc, int64_t strideC, int mode, int64_t idx) {
  const int64_t b = idx / (n * n), rc = idx % (n * n), i = rc / n, j = rc % n;
  if (i <= j) return;
  const double* src = C + (b * strideC + j * ldc + i) * PL;
  double* dst = C + (b * strideC + i * ldc + j) * PL;
  dst[0] = mode > 0 ? src[0] : -src[0];
  if (PL == 2) dst[1] = mode > 0 ? -src[1] : src[1];
}

}  // namespace gk
}  // namespace rr
