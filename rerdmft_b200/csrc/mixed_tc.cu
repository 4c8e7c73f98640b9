// Split-BF16 exchange on the 5th-generation tensor cores (tcgen05 + TMEM + TMA), RR_PREC_MIXED.
//
// Every FP64 operand x is carried as two BF16 numbers, hi = bf16(x) and lo = bf16(x - hi), and a
// product is formed from three BF16 MMAs with FP32 accumulation in TMEM:
//   x y ~= hi_x hi_y + hi_x lo_y + lo_x hi_y          (relative error ~2^-16; lo_x lo_y dropped)
// Two kernels per exchange build, both on one tcgen05 kernel template:
//   half-transform  Tt[P] (n x nocc) = Bt[P] (n x n) . Ct^T   A = Bt (resident, transposed split copy
//                   of B so that the contraction index is contiguous), B = Ct; the epilogue splits
//                   the FP32 tile into hi/lo BF16 rows of T2D[a][P*nocc + i];
//   exchange        K (n x n) = T2D . T2D^T over k = (P, i), upper tile pairs, split-K partials in
//                   FP32, reduced in FP64 in a fixed order.
// Roles: warp 0 lane 0 issues the TMA ring (SWIZZLE_128B tiles of 64 BF16 along K), warp 1 lane 0
// issues the MMAs, all four warps drain TMEM in the epilogue.  Every wait is bounded.
#include <atomic>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "mixed.cuh"
#include "ri_store.cuh"
#include "umma.cuh"

namespace rr {

namespace {

constexpr int BM = 128;
constexpr int BK = 64;  // BF16 per 128-byte swizzled row
constexpr int A_TILE = BM * BK * 2;  // bytes
constexpr int ERR_MMA_FULL = 1 << 4, ERR_MMA_EMPTY = 1 << 5, ERR_MMA_DONE = 1 << 6;

struct UParams {
  int M, N;           // valid extents of the output tile space (rows of A, rows of B)
  int kblocks;        // total 64-wide K blocks
  int splits;         // split-K factor (mode 1)
  int npairs;         // upper-triangular tile pairs (mode 1)
  int ntn;            // N tiles per row of tiles (mode 1)
  // mode 0 output: T2D hi / lo
  __nv_bfloat16* t_hi;
  __nv_bfloat16* t_lo;
  int64_t t_ld;
  int nocc;
  // mode 1 output: FP32 partial tiles
  float* work;
  int* err;
};

template <int BN, int STAGES, int MODE>
struct UCfg {
  static constexpr int B_TILE = BN * BK * 2;
  static constexpr int STAGE = 2 * A_TILE + 2 * B_TILE;
  static constexpr int TX = STAGE;
  static constexpr int SMEM = STAGES * STAGE + 1024 /*align*/ + 256 /*barriers*/;
  static constexpr int TMEM_COLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
  static_assert(B_TILE % 1024 == 0, "B tile must keep 1024-byte alignment");
};

template <int BN, int STAGES, int MODE>
__global__ void __launch_bounds__(128, 1)
    umma_split_kernel(const __grid_constant__ CUtensorMap mapA_hi, const __grid_constant__ CUtensorMap mapA_lo,
                      const __grid_constant__ CUtensorMap mapB_hi, const __grid_constant__ CUtensorMap mapB_lo,
                      const UParams p) {
  using CF = UCfg<BN, STAGES, MODE>;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * CF::STAGE);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // Tile coordinates.
  int m0, n0, P = 0, kb0 = 0, kb1 = p.kblocks, split = 0, pair = 0;
  if (MODE == 0) {
    m0 = blockIdx.x * BM;
    n0 = 0;
    P = blockIdx.y;
  } else {
    pair = blockIdx.x;
    split = blockIdx.y;
    // pair -> (tm, tn) with tm <= tn, row-major over the upper triangle
    int tm = 0, rem = pair;
    while (rem >= p.ntn - tm) { rem -= p.ntn - tm; ++tm; }
    const int tn = tm + rem;
    m0 = tm * BM;
    n0 = tn * BN;
    const int per = (p.kblocks + p.splits - 1) / p.splits;
    kb0 = split * per;
    kb1 = min(p.kblocks, kb0 + per);
  }
  const int nkb = max(0, kb1 - kb0);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    mbar_init(done, 1);
    fence_barrier_init();
    prefetch_tmap(&mapA_hi);
    prefetch_tmap(&mapA_lo);
    prefetch_tmap(&mapB_hi);
    prefetch_tmap(&mapB_lo);
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, CF::TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  bool dead = false;
  if (warp == 0 && lane == 0) {
    // TMA producer
    for (int i = 0; i < nkb && !dead; ++i) {
      const int s = i % STAGES;
      if (i >= STAGES && !mbar_wait(&empty[s], ((i / STAGES) & 1) ^ 1, p.err, ERR_MMA_EMPTY, dead)) break;
      unsigned char* st = smem + s * CF::STAGE;
      const int kc = (kb0 + i) * BK;
      mbar_arrive_expect_tx(&full[s], CF::TX);
      if (MODE == 0) {
        tma_load_3d(st, &mapA_hi, kc, m0, P, &full[s]);
        tma_load_3d(st + A_TILE, &mapA_lo, kc, m0, P, &full[s]);
      } else {
        tma_load_2d(st, &mapA_hi, kc, m0, &full[s]);
        tma_load_2d(st + A_TILE, &mapA_lo, kc, m0, &full[s]);
      }
      tma_load_2d(st + 2 * A_TILE, &mapB_hi, kc, n0, &full[s]);
      tma_load_2d(st + 2 * A_TILE + CF::B_TILE, &mapB_lo, kc, n0, &full[s]);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    constexpr uint32_t idesc = idesc_bf16_f32(BM, BN);
    for (int i = 0; i < nkb; ++i) {
      const int s = i % STAGES;
      mbar_wait(&full[s], (i / STAGES) & 1, p.err, ERR_MMA_FULL, dead);
      tc_fence_after();
      if (!dead) {
        const uint32_t base = smem_u32(smem + s * CF::STAGE);
        const uint64_t ahi = sdesc_k_sw128(base), alo = sdesc_k_sw128(base + A_TILE);
        const uint64_t bhi = sdesc_k_sw128(base + 2 * A_TILE), blo = sdesc_k_sw128(base + 2 * A_TILE + CF::B_TILE);
#pragma unroll
        for (int k = 0; k < BK / 16; ++k) {
          const uint64_t dk = static_cast<uint64_t>(k * 32) >> 4;  // +32 bytes per 16-element step
          umma_bf16(tmem, ahi + dk, bhi + dk, idesc, (i > 0 || k > 0) ? 1u : 0u);
          umma_bf16(tmem, ahi + dk, blo + dk, idesc, 1u);
          umma_bf16(tmem, alo + dk, bhi + dk, idesc, 1u);
        }
      }
      umma_commit(&empty[s]);  // frees the stage once these MMAs have read it
    }
    umma_commit(done);
  }
  // Epilogue: every warp drains its 32 TMEM lanes (rows m0 + 32 warp + lane).
  __syncwarp();
  bool edead = false;
  if (nkb > 0) mbar_wait(done, 0, p.err, ERR_MMA_DONE, edead);
  tc_fence_after();
  const int row = m0 + warp * 32 + lane;
  const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16);
#pragma unroll
  for (int c0 = 0; c0 < BN; c0 += 16) {
    float v[16];
    if (nkb > 0) {
      tmem_ld16(taddr + c0, v);
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = 0.f;
    }
    if (MODE == 0) {
      if (row < p.M) {
        const int64_t rbase = static_cast<int64_t>(row) * p.t_ld + static_cast<int64_t>(P) * p.nocc;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = c0 + j;
          if (col < p.nocc) {
            const __nv_bfloat16 hi = __float2bfloat16_rn(v[j]);
            const __nv_bfloat16 lo = __float2bfloat16_rn(v[j] - __bfloat162float(hi));
            p.t_hi[rbase + col] = hi;
            p.t_lo[rbase + col] = lo;
          }
        }
      }
    } else {
      float* w = p.work + (static_cast<int64_t>(split) * p.npairs + pair) * (BM * BN) + (warp * 32 + lane) * BN + c0;
#pragma unroll
      for (int j = 0; j < 16; ++j) w[j] = v[j];
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, CF::TMEM_COLS);
}

// Persistent half-transform: one CTA per SM walks the (P, 128-row tile) items round robin with one
// continuous TMA ring across items and two TMEM accumulators, so the epilogue of item j (TMEM ->
// split BF16 rows of T2D) overlaps the MMAs of item j + 1.  Roles: warps 0-3 drain TMEM (lanes
// 32 w .. 32 w + 31) and write T2D, warp 4 lane 0 issues the TMA ring, warp 5 lane 0 the MMAs.
// Barriers: full / empty per ring stage, tfull / tempty per accumulator (MMA commit -> epilogue,
// four epilogue warps -> MMA), mdone (all MMAs retired) before TMEM is released.  All waits bounded.
constexpr int HT_THREADS = 192;
constexpr int ERR_HT_FULL = 1 << 7, ERR_HT_EMPTY = 1 << 8, ERR_HT_TFULL = 1 << 9, ERR_HT_TEMPTY = 1 << 10,
              ERR_HT_DONE = 1 << 11;

template <int BN, int STAGES>
struct HCfg {
  static constexpr int B_TILE = BN * BK * 2;
  static constexpr int STAGE = 2 * A_TILE + 2 * B_TILE;
  static constexpr int BNP = BN <= 32 ? 32 : (BN <= 64 ? 64 : 128);  // TMEM columns per accumulator
  static constexpr int TMEM_COLS = 2 * BNP <= 64 ? 64 : (2 * BNP <= 128 ? 128 : 256);
  static constexpr int SMEM = STAGES * STAGE + 1024 + 256;
  static_assert(B_TILE % 1024 == 0, "B tile must keep 1024-byte alignment");
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 128, "UMMA N for M = 128");
};

template <int BN, int STAGES>
__global__ void __launch_bounds__(HT_THREADS, 1)
    umma_ht_persistent_kernel(const __grid_constant__ CUtensorMap mapA_hi, const __grid_constant__ CUtensorMap mapA_lo,
                              const __grid_constant__ CUtensorMap mapB_hi, const __grid_constant__ CUtensorMap mapB_lo,
                              const UParams p, int mtiles, int naux) {
  using CF = HCfg<BN, STAGES>;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * CF::STAGE);
  uint64_t* empty = full + STAGES;
  uint64_t* tfull = empty + STAGES;
  uint64_t* tempty = tfull + 2;
  uint64_t* mdone = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mdone + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t total = static_cast<int64_t>(mtiles) * naux;
  const int nkb = p.kblocks;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    for (int b = 0; b < 2; ++b) { mbar_init(&tfull[b], 1); mbar_init(&tempty[b], 4); }
    mbar_init(mdone, 1);
    fence_barrier_init();
    prefetch_tmap(&mapA_hi);
    prefetch_tmap(&mapA_lo);
    prefetch_tmap(&mapB_hi);
    prefetch_tmap(&mapB_lo);
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, CF::TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  bool dead = false;

  if (warp == 4) {
    if (lane == 0) {  // TMA producer
      uint32_t q = 0;
      for (int64_t item = blockIdx.x; item < total && !dead; item += gridDim.x) {
        const int P = static_cast<int>(item / mtiles), m0 = static_cast<int>(item % mtiles) * BM;
        for (int k = 0; k < nkb; ++k, ++q) {
          const int s = q % STAGES;
          if (q >= STAGES && !mbar_wait(&empty[s], ((q / STAGES) & 1) ^ 1, p.err, ERR_HT_EMPTY, dead)) break;
          unsigned char* st = smem + s * CF::STAGE;
          const int kc = k * BK;
          mbar_arrive_expect_tx(&full[s], CF::STAGE);
          tma_load_3d(st, &mapA_hi, kc, m0, P, &full[s]);
          tma_load_3d(st + A_TILE, &mapA_lo, kc, m0, P, &full[s]);
          tma_load_2d(st + 2 * A_TILE, &mapB_hi, kc, 0, &full[s]);
          tma_load_2d(st + 2 * A_TILE + CF::B_TILE, &mapB_lo, kc, 0, &full[s]);
        }
      }
    }
  } else if (warp == 5) {
    if (lane == 0) {  // MMA issuer
      constexpr uint32_t idesc = idesc_bf16_f32(BM, BN);
      uint32_t q = 0, j = 0;
      for (int64_t item = blockIdx.x; item < total; item += gridDim.x, ++j) {
        const uint32_t b = j & 1;
        if (j >= 2) mbar_wait(&tempty[b], ((j >> 1) - 1) & 1, p.err, ERR_HT_TEMPTY, dead);
        tc_fence_after();
        const uint32_t d = tmem + b * CF::BNP;
        for (int k = 0; k < nkb; ++k, ++q) {
          const int s = q % STAGES;
          mbar_wait(&full[s], (q / STAGES) & 1, p.err, ERR_HT_FULL, dead);
          tc_fence_after();
          if (!dead) {
            const uint32_t base = smem_u32(smem + s * CF::STAGE);
            const uint64_t ahi = sdesc_k_sw128(base), alo = sdesc_k_sw128(base + A_TILE);
            const uint64_t bhi = sdesc_k_sw128(base + 2 * A_TILE), blo = sdesc_k_sw128(base + 2 * A_TILE + CF::B_TILE);
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
              const uint64_t dk = static_cast<uint64_t>(kk * 32) >> 4;
              umma_bf16(d, ahi + dk, bhi + dk, idesc, (k > 0 || kk > 0) ? 1u : 0u);
              umma_bf16(d, ahi + dk, blo + dk, idesc, 1u);
              umma_bf16(d, alo + dk, bhi + dk, idesc, 1u);
            }
          }
          umma_commit(&empty[s]);
        }
        umma_commit(&tfull[b]);
        if (dead) break;
      }
      umma_commit(mdone);
    }
  } else {  // epilogue warps 0-3
    uint32_t j = 0;
    const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
    for (int64_t item = blockIdx.x; item < total; item += gridDim.x, ++j) {
      const uint32_t b = j & 1;
      const bool ok = mbar_wait(&tfull[b], (j >> 1) & 1, p.err, ERR_HT_TFULL, dead);
      tc_fence_after();
      float v[BN];
      if (ok) {
#pragma unroll
        for (int c0 = 0; c0 < BN; c0 += 16) tmem_ld16(tmem + lane_base + b * CF::BNP + c0, v + c0);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[b]);
      if (!ok) break;
      const int P = static_cast<int>(item / mtiles), m0 = static_cast<int>(item % mtiles) * BM;
      const int row = m0 + warp * 32 + lane;
      if (row < p.M) {
        const int64_t rbase = static_cast<int64_t>(row) * p.t_ld + static_cast<int64_t>(P) * p.nocc;
        if ((p.nocc & 7) == 0 && (p.t_ld & 7) == 0) {
          // 16-byte stores: rbase is a multiple of 8 elements when nocc and the row pitch are
#pragma unroll
          for (int c = 0; c < BN; c += 8) {
            if (c < p.nocc) {
              uint32_t h[4], l[4];
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                const __nv_bfloat16 h0 = __float2bfloat16_rn(v[c + 2 * e]), h1 = __float2bfloat16_rn(v[c + 2 * e + 1]);
                const __nv_bfloat16 l0 = __float2bfloat16_rn(v[c + 2 * e] - __bfloat162float(h0));
                const __nv_bfloat16 l1 = __float2bfloat16_rn(v[c + 2 * e + 1] - __bfloat162float(h1));
                h[e] = static_cast<uint32_t>(__bfloat16_as_ushort(h0)) | (static_cast<uint32_t>(__bfloat16_as_ushort(h1)) << 16);
                l[e] = static_cast<uint32_t>(__bfloat16_as_ushort(l0)) | (static_cast<uint32_t>(__bfloat16_as_ushort(l1)) << 16);
              }
              *reinterpret_cast<uint4*>(p.t_hi + rbase + c) = make_uint4(h[0], h[1], h[2], h[3]);
              *reinterpret_cast<uint4*>(p.t_lo + rbase + c) = make_uint4(l[0], l[1], l[2], l[3]);
            }
          }
        } else {
#pragma unroll
          for (int c = 0; c < BN; ++c) {
            if (c < p.nocc) {
              const __nv_bfloat16 hi = __float2bfloat16_rn(v[c]);
              p.t_hi[rbase + c] = hi;
              p.t_lo[rbase + c] = __float2bfloat16_rn(v[c] - __bfloat162float(hi));
            }
          }
        }
      }
    }
  }
  __syncthreads();
  if (warp == 0) {
    bool ddead = false;
    mbar_wait(mdone, 0, p.err, ERR_HT_DONE, ddead);  // every MMA retired before TMEM is released
    tc_fence_after();
    tmem_dealloc(tmem, CF::TMEM_COLS);
  }
}

// Fixed-order reduction of the split-K partial tiles into K (FP64), mirrored to the lower
// triangle: K[a][b] = sum_s work[s][pair(a,b)][a % BM][b % BN].
template <int BN>
__global__ void umma_reduce_kernel(const float* work, int splits, int npairs, int ntn, int n, double alpha, double* K) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < static_cast<int64_t>(n) * n;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int a = static_cast<int>(idx / n), b = static_cast<int>(idx % n);
    const int i = min(a, b), j = max(a, b);  // value from the upper triangle
    const int tm = i / BM, tn = j / BN;
    // pair index of (tm, tn), tm <= tn: sum_{r < tm} (ntn - r) + (tn - tm)
    const int pair = tm * ntn - tm * (tm - 1) / 2 + (tn - tm);
    const int64_t off = static_cast<int64_t>(pair) * (BM * BN) + (i - tm * BM) * BN + (j - tn * BN);
    double s = 0.0;
    for (int sp = 0; sp < splits; ++sp) s += static_cast<double>(work[static_cast<int64_t>(sp) * npairs * (BM * BN) + off]);
    K[idx] = alpha * s;
  }
}

// ---- FP64 -> split BF16 conversions ----

// Bt_hi/lo[P][a][q] (row pitch ldq) from B[P][q][a] (row pitch `pitch` per P, n x n row-major).
__global__ void split_transpose_kernel(const double* B, int64_t pitch, int n, int64_t naux, int ldq, __nv_bfloat16* hi,
                                       __nv_bfloat16* lo) {
  __shared__ double tile[32][33];
  const int tiles = (n + 31) / 32;
  for (int64_t t = blockIdx.x; t < naux * tiles * tiles; t += gridDim.x) {
    const int64_t P = t / (tiles * tiles);
    const int rem = static_cast<int>(t % (tiles * tiles));
    const int q0 = (rem / tiles) * 32, a0 = (rem % tiles) * 32;
    const double* bp = B + P * pitch;
    for (int r = threadIdx.y; r < 32; r += 8) {
      const int q = q0 + r, a = a0 + threadIdx.x;
      tile[r][threadIdx.x] = (q < n && a < n) ? bp[static_cast<int64_t>(q) * n + a] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) {
      const int a = a0 + r, q = q0 + threadIdx.x;
      if (a < n && q < n) {
        const double x = tile[threadIdx.x][r];
        const __nv_bfloat16 h = __double2bfloat16(x);
        const __nv_bfloat16 l = __double2bfloat16(x - static_cast<double>(__bfloat162float(h)));
        const int64_t o = (P * n + a) * ldq + q;
        hi[o] = h;
        lo[o] = l;
      }
    }
    __syncthreads();
  }
}

// Row-major rows x cols FP64 -> split BF16 with row pitch ld.
__global__ void split_rows_bf16_kernel(const double* X, int rows, int cols, int ldx, int ld, __nv_bfloat16* hi,
                                       __nv_bfloat16* lo) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < static_cast<int64_t>(rows) * cols;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(idx / cols), c = static_cast<int>(idx % cols);
    const double x = X[static_cast<int64_t>(r) * ldx + c];
    const __nv_bfloat16 h = __double2bfloat16(x);
    hi[static_cast<int64_t>(r) * ld + c] = h;
    lo[static_cast<int64_t>(r) * ld + c] = __double2bfloat16(x - static_cast<double>(__bfloat162float(h)));
  }
}

// ---- tensor maps through the driver entry point (no libcuda link dependency) ----
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  RR_REQUIRE(fn != nullptr, RR_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  return fn;
}

// BF16 tensor map, innermost dimension first.  dims / strides (bytes, rank-1 entries) / box.
CUtensorMap make_map(const void* base, int rank, const uint64_t* dims, const uint64_t* strides_bytes, const uint32_t* box) {
  CUtensorMap m;
  uint32_t elem[3] = {1, 1, 1};
  const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, static_cast<cuuint32_t>(rank), const_cast<void*>(base),
                                 reinterpret_cast<const cuuint64_t*>(dims), reinterpret_cast<const cuuint64_t*>(strides_bytes),
                                 reinterpret_cast<const cuuint32_t*>(box), reinterpret_cast<const cuuint32_t*>(elem),
                                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  RR_REQUIRE(r == CUDA_SUCCESS, RR_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(static_cast<int>(r)) + ")");
  return m;
}

int sm_count() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

template <int BN, int STAGES, int MODE>
void launch_umma(const CUtensorMap& a_hi, const CUtensorMap& a_lo, const CUtensorMap& b_hi, const CUtensorMap& b_lo,
                 const UParams& p, dim3 grid, cudaStream_t s) {
  using CF = UCfg<BN, STAGES, MODE>;
  auto k = umma_split_kernel<BN, STAGES, MODE>;
  static std::atomic<bool> attr{false};  // host threads may race here: the attribute is idempotent
  if (!attr) {
    RR_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, CF::SMEM));
    attr = true;
  }
  k<<<grid, 128, CF::SMEM, s>>>(a_hi, a_lo, b_hi, b_lo, p);
  RR_LAUNCH_CHECK();
}

int64_t round8(int64_t x) { return (x + 7) / 8 * 8; }

}  // namespace

// Resident split copy of B for the mixed path: Bt_hi/lo[P][a][q], row pitch ldq = round8(n).
void mixed_prepare(MixedOperands& mo, const double* B, int64_t pitch, int64_t n, int64_t naux, cudaStream_t s) {
  if (mo.ready && mo.n == n && mo.naux == naux) return;
  mo.n = n;
  mo.naux = naux;
  mo.ldq = round8(n);
  const int64_t cnt = std::max<int64_t>(naux * n * mo.ldq, 1);
  mo.bt_hi.alloc(static_cast<size_t>(cnt));
  mo.bt_lo.alloc(static_cast<size_t>(cnt));
  RR_CUDA(cudaMemsetAsync(mo.bt_hi.p, 0, sizeof(uint16_t) * cnt, s));
  RR_CUDA(cudaMemsetAsync(mo.bt_lo.p, 0, sizeof(uint16_t) * cnt, s));
  if (naux * n > 0) {
    const int tiles = static_cast<int>((n + 31) / 32);
    const int64_t work = naux * tiles * tiles;
    split_transpose_kernel<<<static_cast<int>(std::min<int64_t>(work, 8LL * sm_count())), dim3(32, 8), 0, s>>>(
        B, pitch, static_cast<int>(n), naux, static_cast<int>(mo.ldq), reinterpret_cast<__nv_bfloat16*>(mo.bt_hi.p),
        reinterpret_cast<__nv_bfloat16*>(mo.bt_lo.p));
    RR_LAUNCH_CHECK();
  }
  mo.ready = true;
}

// K (n x n, FP64, symmetric) = sum_P (Ct B^P)^T (Ct B^P) in split BF16 on tcgen05.
// Ct: nocc x n FP64 row-major (leading dim ldct), device.  Requires nocc <= 48 per pass; larger
// occupied blocks are processed in slices of 48 rows whose contributions add.
void mixed_exchange(MixedOperands& mo, const double* Ct, int64_t ldct, int64_t nocc, double* K, int* err, cudaStream_t s) {
  const int64_t n = mo.n, naux = mo.naux;
  RR_REQUIRE(mo.ready, RR_ERR_STATE, "mixed exchange: operands not prepared");
  RR_REQUIRE(n <= 65535 && naux <= 65535, RR_ERR_ARG, "mixed exchange: dimensions exceed the grid limits");
  if (nocc == 0 || naux == 0 || n == 0) {
    RR_CUDA(cudaMemsetAsync(K, 0, sizeof(double) * n * n, s));
    return;
  }
  constexpr int HT_BN = 48, SY_BN = 128;
  const int64_t ldq = mo.ldq;
  bool first = true;
  for (int64_t i0 = 0; i0 < nocc; i0 += HT_BN) {
    const int64_t r = std::min<int64_t>(HT_BN, nocc - i0);
    // Ct slice -> split BF16 rows (pitch ldq)
    mo.ct_hi.ensure(static_cast<size_t>(HT_BN * ldq));
    mo.ct_lo.ensure(static_cast<size_t>(HT_BN * ldq));
    RR_CUDA(cudaMemsetAsync(mo.ct_hi.p, 0, sizeof(uint16_t) * HT_BN * ldq, s));
    RR_CUDA(cudaMemsetAsync(mo.ct_lo.p, 0, sizeof(uint16_t) * HT_BN * ldq, s));
    split_rows_bf16_kernel<<<static_cast<int>(std::min<int64_t>((r * n + 255) / 256, 1184)), 256, 0, s>>>(
        Ct + i0 * ldct, static_cast<int>(r), static_cast<int>(n), static_cast<int>(ldct), static_cast<int>(ldq),
        reinterpret_cast<__nv_bfloat16*>(mo.ct_hi.p), reinterpret_cast<__nv_bfloat16*>(mo.ct_lo.p));
    RR_LAUNCH_CHECK();
    // T2D rows: (P, i) contiguous per a; pitch rounded to 8 for TMA
    const int64_t kt = naux * r, ldt = round8(kt);
    mo.t_hi.ensure(static_cast<size_t>(n * ldt));
    mo.t_lo.ensure(static_cast<size_t>(n * ldt));
    {
      uint64_t dimsA[3] = {static_cast<uint64_t>(n), static_cast<uint64_t>(n), static_cast<uint64_t>(naux)};
      uint64_t strA[2] = {static_cast<uint64_t>(ldq) * 2, static_cast<uint64_t>(n * ldq) * 2};
      uint32_t boxA[3] = {BK, BM, 1};
      const CUtensorMap a_hi = make_map(mo.bt_hi.p, 3, dimsA, strA, boxA);
      const CUtensorMap a_lo = make_map(mo.bt_lo.p, 3, dimsA, strA, boxA);
      uint64_t dimsB[2] = {static_cast<uint64_t>(n), static_cast<uint64_t>(r)};
      uint64_t strB[1] = {static_cast<uint64_t>(ldq) * 2};
      uint32_t boxB[2] = {BK, HT_BN};
      const CUtensorMap b_hi = make_map(mo.ct_hi.p, 2, dimsB, strB, boxB);
      const CUtensorMap b_lo = make_map(mo.ct_lo.p, 2, dimsB, strB, boxB);
      UParams p{};
      p.M = static_cast<int>(n);
      p.N = static_cast<int>(r);
      p.kblocks = static_cast<int>((n + BK - 1) / BK);
      p.splits = 1;
      p.t_hi = reinterpret_cast<__nv_bfloat16*>(mo.t_hi.p);
      p.t_lo = reinterpret_cast<__nv_bfloat16*>(mo.t_lo.p);
      p.t_ld = ldt;
      p.nocc = static_cast<int>(r);
      p.err = err;
      // Columns [kt, ldt) of T2D are row padding for TMA alignment; the maps' extents stop at kt,
      // so they are never read.
      const int mtiles = static_cast<int>((n + BM - 1) / BM);
      using HC = HCfg<HT_BN, 4>;
      auto kern = umma_ht_persistent_kernel<HT_BN, 4>;
      static std::atomic<bool> attr{false};  // host threads may race here: the attribute is idempotent
      if (!attr) {
        RR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, HC::SMEM));
        attr = true;
      }
      const int64_t items = static_cast<int64_t>(mtiles) * naux;
      const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(items, sm_count())));
      kern<<<grid, HT_THREADS, HC::SMEM, s>>>(a_hi, a_lo, b_hi, b_lo, p, mtiles, static_cast<int>(naux));
      RR_LAUNCH_CHECK();
    }
    {
      uint64_t dims[2] = {static_cast<uint64_t>(kt), static_cast<uint64_t>(n)};
      uint64_t str[1] = {static_cast<uint64_t>(ldt) * 2};
      uint32_t boxA[2] = {BK, BM};
      uint32_t boxB[2] = {BK, SY_BN};
      const CUtensorMap a_hi = make_map(mo.t_hi.p, 2, dims, str, boxA);
      const CUtensorMap a_lo = make_map(mo.t_lo.p, 2, dims, str, boxA);
      const CUtensorMap b_hi = make_map(mo.t_hi.p, 2, dims, str, boxB);
      const CUtensorMap b_lo = make_map(mo.t_lo.p, 2, dims, str, boxB);
      const int ntn = static_cast<int>((n + SY_BN - 1) / SY_BN);
      const int npairs = ntn * (ntn + 1) / 2;  // BM == SY_BN: square tiles
      const int kblocks = static_cast<int>((kt + BK - 1) / BK);
      int splits = std::max(1, std::min(kblocks, static_cast<int>((2LL * sm_count() + npairs - 1) / npairs)));
      const int per = (kblocks + splits - 1) / splits;
      splits = (kblocks + per - 1) / per;
      mo.work.ensure(static_cast<size_t>(static_cast<int64_t>(splits) * npairs * BM * SY_BN));
      UParams p{};
      p.M = static_cast<int>(n);
      p.N = static_cast<int>(n);
      p.kblocks = kblocks;
      p.splits = splits;
      p.npairs = npairs;
      p.ntn = ntn;
      p.work = mo.work.p;
      p.err = err;
      launch_umma<SY_BN, 3, 1>(a_hi, a_lo, b_hi, b_lo, p, dim3(static_cast<unsigned>(npairs), static_cast<unsigned>(splits)),
                                s);
      double* dst = K;
      if (!first) {
        mo.kacc.ensure(static_cast<size_t>(n * n));
        dst = mo.kacc.p;
      }
      umma_reduce_kernel<SY_BN><<<static_cast<int>(std::min<int64_t>((n * n + 255) / 256, 1184)), 256, 0, s>>>(
          mo.work.p, splits, npairs, ntn, static_cast<int>(n), 1.0, dst);
      RR_LAUNCH_CHECK();
      if (!first) axpby(K, dst, 1.0, 1.0, n * n, s);
    }
    first = false;
  }
}

}  // namespace rr
