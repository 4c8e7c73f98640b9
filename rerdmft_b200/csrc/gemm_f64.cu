// FP64 DMMA GEMM: multistage cp.async pipeline (3 stages of 16-deep k tiles), warp tiles of
// (MT*8) x (NT*8) built from mma.sync.m8n8k4.f64, optional complex (4M) accumulation, split-K
// with a fixed-order reduction (bit-identical results run to run), and upper-triangle-only
// scheduling for symmetric / Hermitian outputs.
#include <atomic>
#include <cstdlib>

#include "gemm_f64.cuh"

namespace rr {
namespace {

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
  int mirror;  // split-K reduce of an upper-only product also writes the strict lower triangle (+1 / -1)
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
template <int MT, int NT, int WM, int WN, bool AK, bool BKM, bool CPLX, int V, bool EDOT = false>
__global__ void __launch_bounds__(32 * WM * WN) dgemm_kernel(const Params p) {
  using CF = Cfg<MT, NT, WM, WN, AK, BKM, CPLX>;
  constexpr int BM = CF::BM, BN = CF::BN, THREADS = CF::THREADS, PL = CF::PL;
  extern __shared__ __align__(16) double smem[];

  const int64_t n0 = static_cast<int64_t>(blockIdx.x) * BN;
  const int64_t m0 = static_cast<int64_t>(blockIdx.y) * BM;
  if (p.upper_only && m0 > n0 + BN - 1) return;
  const int64_t bz = blockIdx.z;
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
      p.eout[b * (gridDim.x * gridDim.y) + blockIdx.y * gridDim.x + blockIdx.x] = p.escale * tsum;
    }
  }
}

// Fixed-order split-K reduction: C = alpha * sum_s work[b, s] + beta * C.
template <int PL>
__global__ void splitk_reduce_kernel(const Params p) {
  const int64_t total = p.batch * p.M * p.N;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t b = idx / (p.M * p.N);
    const int64_t rc = idx % (p.M * p.N);
    const int64_t row = rc / p.N, col = rc % p.N;
    if (p.upper_only && row > col) continue;  // written as the mirror of (col, row)
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
    if (p.upper_only && row < col) {
      // the strict lower triangle from the final upper value (mirror requires no plane split and a
      // unit column stride; the lower triangle is never read as beta input here)
      double* t = p.C + (b * p.strideC + col * p.ldc + row) * PL;
      t[0] = p.mirror > 0 ? v[0] : -v[0];
      if (PL == 2) t[1] = p.mirror > 0 ? -v[PL - 1] : v[PL - 1];
    }
  }
}

// Strict lower triangle from the upper one.
template <int PL>
__global__ void mirror_kernel(double* C, int64_t n, int64_t ldc, int64_t strideC, int64_t batch, int mode) {
  const int64_t total = batch * n * n;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t b = idx / (n * n), rc = idx % (n * n), i = rc / n, j = rc % n;
    if (i <= j) continue;
    const double* src = C + (b * strideC + j * ldc + i) * PL;
    double* dst = C + (b * strideC + i * ldc + j) * PL;
    if (PL == 1) {
      dst[0] = mode > 0 ? src[0] : -src[0];
    } else {
      dst[0] = mode > 0 ? src[0] : -src[0];
      dst[1] = mode > 0 ? -src[1] : src[1];
    }
  }
}

int num_sms() { return sm_count_current(); }

template <int MT, int NT, int WM, int WN, bool AK, bool BKM, bool CPLX, int V, bool EDOT = false>
void launch_cfg_v(const Params& p, dim3 grid, cudaStream_t s) {
  using CF = Cfg<MT, NT, WM, WN, AK, BKM, CPLX>;
  auto kern = dgemm_kernel<MT, NT, WM, WN, AK, BKM, CPLX, V, EDOT>;
  static std::atomic<bool> attr[kMaxDevices];
  once_per_device(attr, [&] {
    RR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, CF::SMEM_BYTES));
    // Largest shared-memory carveout: an SM only takes CTAs of another kernel when its carveout
    // fits them too, and the J passes run beside the exchange SYRK.
    RR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
  });
  kern<<<grid, CF::THREADS, CF::SMEM_BYTES, s>>>(p);
  RR_LAUNCH_CHECK();
}

// 16-byte loads need: real data, 16-byte aligned bases and batch strides, even leading dims and
// even contiguous extents (so a pair never straddles the end of a row).
bool vec2_ok(const Params& p, bool AK, bool BKM) {
  auto al = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15) == 0; };
  const bool a = al(p.A) && p.lda % 2 == 0 && p.strideA % 2 == 0 && (AK ? p.K % 2 == 0 : p.M % 2 == 0);
  const bool b = al(p.B) && p.ldb % 2 == 0 && p.strideB % 2 == 0 && (BKM ? p.K % 2 == 0 : p.N % 2 == 0);
  return a && b && p.kchunk % 2 == 0;
}

template <int MT, int NT, int WM, int WN, bool AK, bool BKM, bool CPLX>
void launch_cfg(const Params& p, dim3 grid, cudaStream_t s) {
  if constexpr (!CPLX && AK && !BKM) {  // the half-transform layout is the only one with an epilogue dot
    if (p.eout) {
      if (vec2_ok(p, AK, BKM)) return launch_cfg_v<MT, NT, WM, WN, AK, BKM, CPLX, 2, true>(p, grid, s);
      return launch_cfg_v<MT, NT, WM, WN, AK, BKM, CPLX, 1, true>(p, grid, s);
    }
  }
  if constexpr (!CPLX) {
    if (vec2_ok(p, AK, BKM)) return launch_cfg_v<MT, NT, WM, WN, AK, BKM, CPLX, 2>(p, grid, s);
  }
  launch_cfg_v<MT, NT, WM, WN, AK, BKM, CPLX, 1>(p, grid, s);
}

struct Shape { int bm, bn; };

// Square tiles for M > 48: 80 x 80 (5 x 5 fragments per warp) for long-K products (the exchange
// SYRK) when it covers M x N with less padding than 64 x 64 (n = 400: 400^2 instead of 448^2
// computed); short-K products keep 64 x 64, whose larger CTA count hides their latency better.
bool use_tile80(int64_t M, int64_t N, int64_t K) {
  const int64_t p64 = static_cast<int64_t>(ceil_div(M, 64)) * 64 * ceil_div(N, 64) * 64;
  const int64_t p80 = static_cast<int64_t>(ceil_div(M, 80)) * 80 * ceil_div(N, 80) * 80;
  return K >= 8192 && p80 < p64;
}

// Batched half-transforms of 49..128 coefficient rows (the relativistic [Re; Im] rows, 2 r = 80 at
// 40 spinors): the batch fills the GPU at any tile size, so the tile that pads M x N least wins;
// 80 x 80 when it pads less than 64 x 64 and 32 x 32 (80 x 600: 80 x 640 instead of 128 x 640).
bool batched_tile80(int64_t M, int64_t N, int64_t batch) {
  if (M <= 48 || M > 128 || batch < num_sms()) return false;
  auto pad = [&](int64_t t) { return static_cast<int64_t>(ceil_div(M, t)) * t * ceil_div(N, t) * t; };
  return pad(80) < pad(64) && pad(80) < pad(32);
}

// Small square products (SP2 purification, DIIS, recovery at n <= 512): 32 x 32 tiles without
// split-K: more CTAs and no reduction launch; measured 14 us instead of 20 us at n = 400.
bool use_tile32(int64_t M, int64_t N, int64_t K) { return M > 48 && M <= 512 && N <= 512 && K <= 2048; }

template <bool AK, bool BKM>
void launch_real(const Params& p, dim3 grid, cudaStream_t s) {
  if (batched_tile80(p.M, p.N, p.batch)) return launch_cfg<5, 5, 2, 2, AK, BKM, false>(p, grid, s);
  if (use_tile32(p.M, p.N, p.K)) return launch_cfg<2, 2, 2, 2, AK, BKM, false>(p, grid, s);
  if (p.M <= 48) {
    switch ((p.M + 7) / 8) {
      case 1: return launch_cfg<1, 4, 1, 4, AK, BKM, false>(p, grid, s);
      case 2: return launch_cfg<2, 4, 1, 4, AK, BKM, false>(p, grid, s);
      case 3: return launch_cfg<3, 4, 1, 4, AK, BKM, false>(p, grid, s);
      case 4: return launch_cfg<4, 4, 1, 4, AK, BKM, false>(p, grid, s);
      case 5: return launch_cfg<5, 2, 1, 5, AK, BKM, false>(p, grid, s);  // 40 x 80: see pick_shape
      default: return launch_cfg<6, 4, 1, 4, AK, BKM, false>(p, grid, s);
    }
  }
  if (use_tile80(p.M, p.N, p.K)) return launch_cfg<5, 5, 2, 2, AK, BKM, false>(p, grid, s);
  launch_cfg<4, 4, 2, 2, AK, BKM, false>(p, grid, s);
}

// Complex products: 32 x 32 tiles with K split up to 4 ways up to n = 1024 (measured 97 instead of
// 114 us for a Hermitian 800^3 product, 27 instead of 39 us at 400), 32 x 64 above.
bool cplx_tile32(const GemmDesc& d) { return d.cplx && d.M <= 1024 && d.N <= 1024; }

Shape pick_shape(const GemmDesc& d) {
  if (cplx_tile32(d)) return {32, 32};
  if (d.cplx) return {32, 64};
  if (batched_tile80(d.M, d.N, d.batch)) return {80, 80};
  if (use_tile32(d.M, d.N, d.K)) return {32, 32};
  // 33..40 rows (the half-transform at 40 occupied orbitals): 40 x 80 tiles of five 40 x 16 warps,
  // measured 847 instead of 901 us at n = 400, naux = 1600 (80 divides typical n exactly).
  if (d.M <= 48) return {static_cast<int>(8 * ((d.M + 7) / 8)), (d.M + 7) / 8 == 5 ? 80 : 128};
  if (use_tile80(d.M, d.N, d.K)) return {80, 80};
  return {64, 64};
}

int pick_splits(const GemmDesc& d, Shape sh, int64_t* kchunk) {
  int64_t tiles = static_cast<int64_t>(ceil_div(d.M, sh.bm)) * ceil_div(d.N, sh.bn) * d.batch;
  if (d.mirror) tiles = (tiles + ceil_div(d.M, sh.bm) * d.batch) / 2;
  // Enough CTAs for several waves (load balance across SMs), K chunks of at least 128: eight waves
  // for upper-tile products (the exchange SYRK: 4 or 16 measured slower), sixteen for full ones
  // (the 4c exchange blocks: 24.3 -> 23.5 ms per build against eight).
  const int64_t target = (d.mirror ? 8LL : 16LL) * num_sms();
  int splits = 1;
  if (cplx_tile32(d) || (sh.bm == 32 && sh.bn == 32 && tiles < 2LL * num_sms())) {
    // small square products (recovery, SCF): one wave of 32 x 32 tiles at most, so split K up to 4
    splits = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(4, d.K / (4 * KT))));
  } else if (!(sh.bm == 32 && sh.bn == 32) && tiles < 2LL * num_sms() && d.K >= 8 * KT) {
    splits = static_cast<int>(std::min<int64_t>((target + tiles - 1) / tiles, d.K / (8 * KT)));
    splits = std::max(1, std::min(splits, 128));
  }
  int64_t kc = round_up((d.K + splits - 1) / splits, KT);
  splits = static_cast<int>((d.K + kc - 1) / kc);
  *kchunk = kc;
  return std::max(1, splits);
}

}  // namespace

int64_t gemm_tiles_per_batch(const GemmDesc& d) {
  const Shape sh = pick_shape(d);
  return static_cast<int64_t>(ceil_div(d.N, sh.bn)) * ceil_div(d.M, sh.bm);
}

int64_t gemm_work_doubles(const GemmDesc& d) {
  int64_t kc;
  const int s = pick_splits(d, pick_shape(d), &kc);
  return s > 1 ? d.batch * s * d.M * d.N * (d.cplx ? 2 : 1) : 0;
}

void gemm(const GemmDesc& d, cudaStream_t stream, double* work, int64_t work_cap) {
  RR_REQUIRE(d.M >= 0 && d.N >= 0 && d.K >= 0 && d.batch >= 0, RR_ERR_ARG, "gemm: negative size");
  RR_REQUIRE(!d.mirror || d.M == d.N, RR_ERR_ARG, "gemm: mirror needs a square output");
  RR_REQUIRE(!d.mirror || d.c_plane_rows == 0, RR_ERR_ARG, "gemm: mirror with planar output");
  if (d.M == 0 || d.N == 0 || d.batch == 0) return;
  const Shape sh = pick_shape(d);
  Params p{};
  p.M = d.M; p.N = d.N; p.K = d.K;
  p.A = d.A; p.lda = d.lda; p.strideA = d.strideA;
  p.B = d.B; p.ldb = d.ldb; p.strideB = d.strideB;
  p.C = d.C; p.ldc = d.ldc; p.strideC = d.strideC;
  p.alpha = d.alpha; p.beta = d.beta; p.batch = d.batch;
  p.signA = d.conjA ? -1.0 : 1.0;
  p.signB = d.conjB ? -1.0 : 1.0;
  p.c_plane_rows = d.c_plane_rows; p.c_plane_stride = d.c_plane_stride;
  p.ccs = d.c_col_stride;
  RR_REQUIRE(d.c_col_stride >= 1 && (d.c_col_stride == 1 || !d.cplx), RR_ERR_ARG, "gemm: bad output column stride");
  RR_REQUIRE(d.c_col_stride == 1 || !d.mirror, RR_ERR_ARG, "gemm: mirror with strided output");
  p.upper_only = d.mirror != 0;
  p.mirror = d.mirror;
  p.eE = d.edot_E;
  p.eld = d.edot_ld;
  p.escale = d.edot_scale;
  p.eout = d.edot_out;
  if (d.edot_out) {
    RR_REQUIRE(!d.cplx && d.opA == Op::N && d.opB == Op::N && d.c_plane_rows == 0 && !d.mirror, RR_ERR_ARG,
               "gemm: epilogue dot supports the real N,N layout only");
    work = nullptr;  // one K range per CTA
  }
  int64_t kc = d.K;
  int splits = 1;
  if (work && d.K > 0) {
    splits = pick_splits(d, sh, &kc);
    while (splits > 1 && d.batch * splits * d.M * d.N * (d.cplx ? 2 : 1) > work_cap) {
      splits = (splits + 1) / 2;
      kc = round_up((d.K + splits - 1) / splits, KT);
      splits = static_cast<int>((d.K + kc - 1) / kc);
    }
  }
  if (splits <= 1) { splits = 1; kc = std::max<int64_t>(d.K, 1); }
  p.splits = splits; p.kchunk = kc; p.work = work;
  RR_REQUIRE(d.batch * splits <= 65535, RR_ERR_ARG, "gemm: batch x splits exceeds the grid z limit");
  dim3 grid(ceil_div(d.N, sh.bn), ceil_div(d.M, sh.bm), static_cast<unsigned>(d.batch * splits));
  const bool AK = d.opA == Op::N, BKM = d.opB == Op::T;
  if (cplx_tile32(d)) {
    if (AK && BKM) launch_cfg<2, 2, 2, 2, true, true, true>(p, grid, stream);
    else if (AK) launch_cfg<2, 2, 2, 2, true, false, true>(p, grid, stream);
    else if (BKM) launch_cfg<2, 2, 2, 2, false, true, true>(p, grid, stream);
    else launch_cfg<2, 2, 2, 2, false, false, true>(p, grid, stream);
  } else if (d.cplx) {
    if (AK && BKM) launch_cfg<2, 4, 2, 2, true, true, true>(p, grid, stream);
    else if (AK) launch_cfg<2, 4, 2, 2, true, false, true>(p, grid, stream);
    else if (BKM) launch_cfg<2, 4, 2, 2, false, true, true>(p, grid, stream);
    else launch_cfg<2, 4, 2, 2, false, false, true>(p, grid, stream);
  } else {
    if (AK && BKM) launch_real<true, true>(p, grid, stream);
    else if (AK) launch_real<true, false>(p, grid, stream);
    else if (BKM) launch_real<false, true>(p, grid, stream);
    else launch_real<false, false>(p, grid, stream);
  }
  const int blocks = std::min<int64_t>(4LL * num_sms(), std::max<int64_t>(1, (d.batch * d.M * d.N + 255) / 256));
  if (splits > 1) {
    if (d.cplx) splitk_reduce_kernel<2><<<blocks, 256, 0, stream>>>(p);
    else splitk_reduce_kernel<1><<<blocks, 256, 0, stream>>>(p);
    RR_LAUNCH_CHECK();
  }
  if (d.mirror && splits == 1) {  // with split-K the reduction wrote the mirror
    if (d.cplx) mirror_kernel<2><<<blocks, 256, 0, stream>>>(d.C, d.M, d.ldc, d.strideC, d.batch, d.mirror);
    else mirror_kernel<1><<<blocks, 256, 0, stream>>>(d.C, d.M, d.ldc, d.strideC, d.batch, d.mirror);
    RR_LAUNCH_CHECK();
  }
  // RR_DEBUG_SYNC=1: finish every product before returning and name the one that failed.
  static const bool debug_sync = std::getenv("RR_DEBUG_SYNC") != nullptr;
  if (debug_sync) {
    const cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess)
      throw Error(RR_ERR_CUDA, "gemm M=" + std::to_string(d.M) + " N=" + std::to_string(d.N) + " K=" +
                                   std::to_string(d.K) + " batch=" + std::to_string(d.batch) + " cplx=" +
                                   std::to_string(d.cplx) + " mirror=" + std::to_string(d.mirror) + " opA=" +
                                   std::to_string(static_cast<int>(d.opA)) + " opB=" +
                                   std::to_string(static_cast<int>(d.opB)) + " lda=" + std::to_string(d.lda) +
                                   " ldb=" + std::to_string(d.ldb) + " ldc=" + std::to_string(d.ldc) + " splits=" +
                                   std::to_string(splits) + " kchunk=" + std::to_string(kc) + " tile=" +
                                   std::to_string(sh.bm) + "x" + std::to_string(sh.bn) + " work_cap=" +
                                   std::to_string(work_cap) + ": " + cudaGetErrorString(e));
  }
}

}  // namespace rr
