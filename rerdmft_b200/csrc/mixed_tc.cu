// Split-BF16 exchange on the 5th-generation tensor cores (tcgen05 + TMEM + TMA), RR_PREC_MIXED.
//
// Every FP64 operand x is carried as two BF16 numbers, hi = bf16(x) and lo = bf16(x - hi), and a
// product is formed from three BF16 MMAs with FP32 accumulation in TMEM:
//   x y ~= hi_x hi_y + hi_x lo_y + lo_x hi_y          (relative error ~2^-16; lo_x lo_y dropped)
// Two kernels per exchange build:
//   half-transform  (persistent) for every aux index P and 128-row tile of AO index a:
//                   out[a][j] = sum_q Bt[P][a][q] coef[j][q] over the coefficient rows j of the pass;
//                   the epilogue splits the FP32 tile into hi/lo BF16 and scatters column j into one
//                   or more output planes [a][P*period + j'] (a permutation of the rows with signs),
//                   so that each exchange block below is a plain K-contiguous product;
//   exchange GEMM   K (M x N) = A . B^T over k = (P, j) of two planes, upper tile pairs for a
//                   Hermitian diagonal block, split-K partials in FP32 reduced in FP64 in a fixed
//                   order by the placement kernel, which also mirrors and scatters into K.
// Roles (GEMM): warp 0 lane 0 issues the TMA ring (SWIZZLE_128B tiles of 64 BF16 along K), warp 1
// lane 0 issues the MMAs, all four warps drain TMEM.  Every wait is bounded.
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

// ---- exchange GEMM: K tile (128 x 128) = A rows . B rows^T, split-K partials ----
constexpr int GBN = 128;
constexpr int G_STAGES = 3;

struct GParams {
  int kblocks;  // 64-wide K blocks
  int splits;   // split-K factor
  int tiles;    // output tiles per split
  int ntn;      // N tiles per row of tiles
  int upper;    // 1: tiles are the upper-triangular pairs tm <= tn of a square output
  float* work;  // [split][tile][128][128]
  int* err;
};

struct GCfg {
  static constexpr int B_TILE = GBN * BK * 2;
  static constexpr int STAGE = 2 * A_TILE + 2 * B_TILE;
  static constexpr int SMEM = G_STAGES * STAGE + 1024 /*align*/ + 256 /*barriers*/;
  static constexpr int TMEM_COLS = 128;
};

__global__ void __launch_bounds__(128, 1)
    umma_gemm_kernel(const __grid_constant__ CUtensorMap mapA_hi, const __grid_constant__ CUtensorMap mapA_lo,
                     const __grid_constant__ CUtensorMap mapB_hi, const __grid_constant__ CUtensorMap mapB_lo,
                     const GParams p) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + G_STAGES * GCfg::STAGE);
  uint64_t* empty = full + G_STAGES;
  uint64_t* done = empty + G_STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  const int tile = blockIdx.x, split = blockIdx.y;
  int tm, tn;
  if (p.upper) {  // tile -> (tm, tn), tm <= tn, row-major over the upper triangle
    tm = 0;
    int rem = tile;
    while (rem >= p.ntn - tm) { rem -= p.ntn - tm; ++tm; }
    tn = tm + rem;
  } else {
    tm = tile / p.ntn;
    tn = tile % p.ntn;
  }
  const int m0 = tm * BM, n0 = tn * GBN;
  const int per = (p.kblocks + p.splits - 1) / p.splits;
  const int kb0 = split * per;
  const int nkb = max(0, min(p.kblocks, kb0 + per) - kb0);

  if (threadIdx.x == 0) {
    for (int s = 0; s < G_STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    mbar_init(done, 1);
    fence_barrier_init();
    prefetch_tmap(&mapA_hi);
    prefetch_tmap(&mapA_lo);
    prefetch_tmap(&mapB_hi);
    prefetch_tmap(&mapB_lo);
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, GCfg::TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  bool dead = false;
  if (warp == 0 && lane == 0) {  // TMA producer
    for (int i = 0; i < nkb && !dead; ++i) {
      const int s = i % G_STAGES;
      if (i >= G_STAGES && !mbar_wait(&empty[s], ((i / G_STAGES) & 1) ^ 1, p.err, ERR_MMA_EMPTY, dead)) break;
      unsigned char* st = smem + s * GCfg::STAGE;
      const int kc = (kb0 + i) * BK;
      mbar_arrive_expect_tx(&full[s], GCfg::STAGE);
      tma_load_2d(st, &mapA_hi, kc, m0, &full[s]);
      tma_load_2d(st + A_TILE, &mapA_lo, kc, m0, &full[s]);
      tma_load_2d(st + 2 * A_TILE, &mapB_hi, kc, n0, &full[s]);
      tma_load_2d(st + 2 * A_TILE + GCfg::B_TILE, &mapB_lo, kc, n0, &full[s]);
    }
  } else if (warp == 1 && lane == 0) {  // MMA issuer
    constexpr uint32_t idesc = idesc_bf16_f32(BM, GBN);
    for (int i = 0; i < nkb; ++i) {
      const int s = i % G_STAGES;
      mbar_wait(&full[s], (i / G_STAGES) & 1, p.err, ERR_MMA_FULL, dead);
      tc_fence_after();
      if (!dead) {
        const uint32_t base = smem_u32(smem + s * GCfg::STAGE);
        const uint64_t ahi = sdesc_k_sw128(base), alo = sdesc_k_sw128(base + A_TILE);
        const uint64_t bhi = sdesc_k_sw128(base + 2 * A_TILE), blo = sdesc_k_sw128(base + 2 * A_TILE + GCfg::B_TILE);
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
  // Epilogue: every warp drains its 32 TMEM lanes (tile rows 32 warp + lane) into FP32 partials.
  __syncwarp();
  bool edead = false;
  if (nkb > 0) mbar_wait(done, 0, p.err, ERR_MMA_DONE, edead);
  tc_fence_after();
  const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16);
  float* w = p.work + (static_cast<int64_t>(split) * p.tiles + tile) * (BM * GBN) + (warp * 32 + lane) * GBN;
#pragma unroll 2
  for (int c0 = 0; c0 < GBN; c0 += 16) {
    float v[16];
    if (nkb > 0) {
      tmem_ld16(taddr + c0, v);
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = 0.f;
    }
#pragma unroll
    for (int j = 0; j < 16; j += 4) *reinterpret_cast<float4*>(w + c0 + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, GCfg::TMEM_COLS);
}

// Fixed-order reduction of the split-K partial tiles of one exchange block, scattered into K:
// value(a, b) = sum_s work[s][tile(a, b)][a % 128][b % 128] (real part from wre, imaginary part from
// wim when given).  For an upper-tile block the lower triangle takes the mirrored value, with the
// imaginary part negated (Hermitian).  K entry (of + a, ou + b) receives the value; with `both` the
// entry (ou + b, of + a) receives its conjugate.  Complex K is interleaved.
__global__ void umma_place_kernel(const float* wre, const float* wim, int splits, int tiles, int ntn, int upper, int M,
                                  int N, double* K, int64_t ldk, int64_t of, int64_t ou, int both, int accumulate,
                                  int cplx) {
  const int64_t tile_sz = static_cast<int64_t>(BM) * GBN;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < static_cast<int64_t>(M) * N;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int a = static_cast<int>(idx / N), b = static_cast<int>(idx % N);
    int i = a, j = b;
    double sim = 1.0;
    if (upper && a > b) { i = b; j = a; sim = -1.0; }
    const int tm = i / BM, tn = j / GBN;
    const int t = upper ? tm * ntn - tm * (tm - 1) / 2 + (tn - tm) : tm * ntn + tn;
    const int64_t off = static_cast<int64_t>(t) * tile_sz + static_cast<int64_t>(i - tm * BM) * GBN + (j - tn * GBN);
    double re = 0.0, im = 0.0;
    for (int sp = 0; sp < splits; ++sp) re += static_cast<double>(wre[static_cast<int64_t>(sp) * tiles * tile_sz + off]);
    if (wim)
      for (int sp = 0; sp < splits; ++sp) im += static_cast<double>(wim[static_cast<int64_t>(sp) * tiles * tile_sz + off]);
    im = upper && a == b ? 0.0 : im * sim;  // a Hermitian block has a real diagonal
    if (cplx) {
      double* k = K + ((of + a) * ldk + ou + b) * 2;
      k[0] = accumulate ? k[0] + re : re;
      k[1] = accumulate ? k[1] + im : im;
      if (both) {
        double* kt = K + ((ou + b) * ldk + of + a) * 2;
        kt[0] = accumulate ? kt[0] + re : re;
        kt[1] = accumulate ? kt[1] - im : -im;
      }
    } else {
      double* k = K + (of + a) * ldk + ou + b;
      *k = accumulate ? *k + re : re;
      if (both) {
        double* kt = K + (ou + b) * ldk + of + a;
        *kt = accumulate ? *kt + re : re;
      }
    }
  }
}

// K (+)= X + X^dagger over the whole ldk x ldk matrix (real: X + X^T; complex interleaved).
__global__ void herm_add_kernel(double* K, const double* X, int64_t ldk, int accumulate, int cplx) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < ldk * ldk;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx / ldk, j = idx % ldk, t = j * ldk + i;
    if (cplx) {
      const double re = X[2 * idx] + X[2 * t], im = X[2 * idx + 1] - X[2 * t + 1];
      K[2 * idx] = accumulate ? K[2 * idx] + re : re;
      K[2 * idx + 1] = accumulate ? K[2 * idx + 1] + im : im;
    } else {
      const double v = X[idx] + X[t];
      K[idx] = accumulate ? K[idx] + v : v;
    }
  }
}

// ---- persistent half-transform ----
// One CTA per SM walks the (P, 128-row tile) items round robin with one continuous TMA ring across
// items and two TMEM accumulators, so the epilogue of item j (TMEM -> split BF16 planes) overlaps the
// MMAs of item j + 1.  Roles: warps 0-3 drain TMEM (lanes 32 w .. 32 w + 31) and write the planes,
// warp 4 lane 0 issues the TMA ring, warp 5 lane 0 the MMAs.  Barriers: full / empty per ring stage,
// tfull / tempty per accumulator (MMA commit -> epilogue, four epilogue warps -> MMA), mdone (all
// MMAs retired) before TMEM is released.  All waits bounded.
constexpr int HT_THREADS = 192;
constexpr int ERR_HT_FULL = 1 << 7, ERR_HT_EMPTY = 1 << 8, ERR_HT_TFULL = 1 << 9, ERR_HT_TEMPTY = 1 << 10,
              ERR_HT_DONE = 1 << 11;

// Epilogue layout.  The pass's columns form `groups` groups of `period` columns (one flavour each);
// a group is made of blocks of `blk` columns.  Column c of group g, in block q = c / blk, goes to
// plane o of that group at column P * operiod + dst[o][q] * blk + c % blk, multiplied by
// sgn[o][q]; dst[o][q] < 0 leaves block q out of plane o.
struct HtEpi {
  __nv_bfloat16* hi[2][3];
  __nv_bfloat16* lo[2][3];
  int64_t ld;  // row pitch of every plane (elements)
  int ncols, groups, planes, period, operiod, blk;
  signed char dst[3][4], sgn[3][4];
};

template <int BN, int STAGES>
struct HCfg {
  static constexpr int B_TILE = BN * BK * 2;
  static constexpr int STAGE = 2 * A_TILE + 2 * B_TILE;
  static constexpr int BNP = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));  // TMEM columns per accumulator
  static constexpr int TMEM_COLS = 2 * BNP <= 64 ? 64 : (2 * BNP <= 128 ? 128 : (2 * BNP <= 256 ? 256 : 512));
  static constexpr int SMEM = STAGES * STAGE + 1024 + 256;
  static_assert(B_TILE % 1024 == 0, "B tile must keep 1024-byte alignment");
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "UMMA N for M = 128");
  static_assert(SMEM <= 232448, "shared memory per CTA");
};

__device__ __forceinline__ uint32_t pack_bf16(float x, float y) {
  return static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16_rn(x))) |
         (static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16_rn(y))) << 16);
}

// Writes 16 accumulator columns c0 .. c0 + 15 of row `row` (aux index P) into the planes.
__device__ __forceinline__ void ht_store16(const HtEpi& e, int64_t row, int P, int c0, const float* v, bool vec) {
  const int64_t rbase = row * e.ld + static_cast<int64_t>(P) * e.operiod;
  if (vec) {
#pragma unroll
    for (int h8 = 0; h8 < 16; h8 += 8) {
      const int gc = c0 + h8;
      if (gc < e.ncols) {
        const int g = gc / e.period, c = gc - g * e.period, q = c / e.blk, cin = c - q * e.blk;
        for (int o = 0; o < e.planes; ++o) {
          if (e.dst[o][q] < 0) continue;
          const float sg = static_cast<float>(e.sgn[o][q]);
          const int64_t off = rbase + e.dst[o][q] * e.blk + cin;
          uint32_t h[4], l[4];
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const float x0 = sg * v[h8 + 2 * t], x1 = sg * v[h8 + 2 * t + 1];
            const float r0 = __bfloat162float(__float2bfloat16_rn(x0)), r1 = __bfloat162float(__float2bfloat16_rn(x1));
            h[t] = pack_bf16(x0, x1);
            l[t] = pack_bf16(x0 - r0, x1 - r1);
          }
          *reinterpret_cast<uint4*>(e.hi[g][o] + off) = make_uint4(h[0], h[1], h[2], h[3]);
          *reinterpret_cast<uint4*>(e.lo[g][o] + off) = make_uint4(l[0], l[1], l[2], l[3]);
        }
      }
    }
  } else {
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      const int gc = c0 + t;
      if (gc >= e.ncols) continue;
      const int g = gc / e.period, c = gc - g * e.period, q = c / e.blk, cin = c - q * e.blk;
      for (int o = 0; o < e.planes; ++o) {
        if (e.dst[o][q] < 0) continue;
        const float x = static_cast<float>(e.sgn[o][q]) * v[t];
        const __nv_bfloat16 hi = __float2bfloat16_rn(x);
        const int64_t off = rbase + e.dst[o][q] * e.blk + cin;
        e.hi[g][o][off] = hi;
        e.lo[g][o][off] = __float2bfloat16_rn(x - __bfloat162float(hi));
      }
    }
  }
}

template <int BN, int STAGES>
__global__ void __launch_bounds__(HT_THREADS, 1)
    umma_ht_persistent_kernel(const __grid_constant__ CUtensorMap mapA_hi, const __grid_constant__ CUtensorMap mapA_lo,
                              const __grid_constant__ CUtensorMap mapB_hi, const __grid_constant__ CUtensorMap mapB_lo,
                              const __grid_constant__ HtEpi e, int M, int nkb, int mtiles, int naux, int* err) {
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
          if (q >= STAGES && !mbar_wait(&empty[s], ((q / STAGES) & 1) ^ 1, err, ERR_HT_EMPTY, dead)) break;
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
        if (j >= 2) mbar_wait(&tempty[b], ((j >> 1) - 1) & 1, err, ERR_HT_TEMPTY, dead);
        tc_fence_after();
        const uint32_t d = tmem + b * CF::BNP;
        for (int k = 0; k < nkb; ++k, ++q) {
          const int s = q % STAGES;
          mbar_wait(&full[s], (q / STAGES) & 1, err, ERR_HT_FULL, dead);
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
    // 16-byte stores need 8-column runs that stay inside one block and aligned plane columns.
    const bool vec = (e.blk & 7) == 0 && (e.period & 7) == 0 && (e.operiod & 7) == 0 && (e.ncols & 7) == 0 &&
                     (e.ld & 7) == 0;
    for (int64_t item = blockIdx.x; item < total; item += gridDim.x, ++j) {
      const uint32_t b = j & 1;
      const bool ok = mbar_wait(&tfull[b], (j >> 1) & 1, err, ERR_HT_TFULL, dead);
      tc_fence_after();
      if (ok) {
        const int P = static_cast<int>(item / mtiles), m0 = static_cast<int>(item % mtiles) * BM;
        const int row = m0 + warp * 32 + lane;
        for (int c0 = 0; c0 < BN && c0 < e.ncols; c0 += 16) {  // c0 is warp-uniform
          float v[16];
          tmem_ld16(tmem + lane_base + b * CF::BNP + c0, v);
          if (row < M) ht_store16(e, row, P, c0, v, vec);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[b]);
      if (!ok) break;
    }
  }
  __syncthreads();
  if (warp == 0) {
    bool ddead = false;
    mbar_wait(mdone, 0, err, ERR_HT_DONE, ddead);  // every MMA retired before TMEM is released
    tc_fence_after();
    tmem_dealloc(tmem, CF::TMEM_COLS);
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

// Coefficient rows of one half-transform pass, split into BF16 hi/lo rows of pitch ldq.  Group g
// (flavour columns [off_g, off_g + fs) of c_t) spans nblk * r8 rows; row q * r8 + i of the group
// holds, for slice row i0 + i of c_t (zero when i >= rs):
//   mode 0 (real):                  Ct
//   mode 1 (real, incremental):     W, U
//   mode 2 (complex):               Re Ct, Im Ct
//   mode 3 (complex, incremental):  Re W, Im W, Re U, Im U
// with W = (Ct + Ct_prev) / 2 and U = Ct - Ct_prev.  ld counts scalars (real) or complex entries.
__global__ void coef_rows_kernel(const double* Ct, const double* Ctp, int64_t ld, int64_t i0, int rs, int r8, int mode,
                                 int groups, int64_t off0, int64_t off1, int fs, int ldq, __nv_bfloat16* hi,
                                 __nv_bfloat16* lo) {
  const int nblk = mode == 0 ? 1 : (mode == 3 ? 4 : 2);
  const int period = nblk * r8;
  const int64_t rows = static_cast<int64_t>(groups) * period;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < rows * fs;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int row = static_cast<int>(idx / fs), a = static_cast<int>(idx % fs);
    const int g = row / period, c = row - g * period, q = c / r8, i = c - q * r8;
    double x = 0.0;
    if (i < rs) {
      const int64_t e = (i0 + i) * ld + (g ? off1 : off0) + a;
      if (mode == 0) {
        x = Ct[e];
      } else if (mode == 1) {
        x = q == 0 ? 0.5 * (Ct[e] + Ctp[e]) : Ct[e] - Ctp[e];
      } else if (mode == 2) {
        x = Ct[2 * e + q];
      } else {
        const int part = q & 1;
        const double cur = Ct[2 * e + part], prv = Ctp[2 * e + part];
        x = q < 2 ? 0.5 * (cur + prv) : cur - prv;
      }
    }
    const __nv_bfloat16 h = __double2bfloat16(x);
    hi[static_cast<int64_t>(row) * ldq + a] = h;
    lo[static_cast<int64_t>(row) * ldq + a] = __double2bfloat16(x - static_cast<double>(__bfloat162float(h)));
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

int sm_count() { return sm_count_current(); }

int64_t round8(int64_t x) { return (x + 7) / 8 * 8; }
int grid_for(int64_t count) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((count + 255) / 256, 1184))); }

template <int BN, int STAGES>
void launch_ht_bn(const CUtensorMap& a_hi, const CUtensorMap& a_lo, const CUtensorMap& b_hi, const CUtensorMap& b_lo,
                  const HtEpi& e, int M, int nkb, int mtiles, int naux, int* err, cudaStream_t s) {
  using HC = HCfg<BN, STAGES>;
  auto kern = umma_ht_persistent_kernel<BN, STAGES>;
  static std::atomic<bool> attr[kMaxDevices];
  once_per_device(attr, [&] { RR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, HC::SMEM)); });
  const int64_t items = static_cast<int64_t>(mtiles) * naux;
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(items, sm_count())));
  kern<<<grid, HT_THREADS, HC::SMEM, s>>>(a_hi, a_lo, b_hi, b_lo, e, M, nkb, mtiles, naux, err);
  RR_LAUNCH_CHECK();
}

// Half-transform pass of tensor `mo` against `rows` coefficient rows (split BF16, pitch mo.ldq);
// the accumulator width is the smallest supported UMMA N >= rows.
void launch_ht(const MixedOperands& mo, const uint16_t* coef_hi, const uint16_t* coef_lo, int rows, const HtEpi& e,
               int* err, cudaStream_t s) {
  const int64_t n = mo.n, naux = mo.naux, ldq = mo.ldq;
  uint64_t dimsA[3] = {static_cast<uint64_t>(n), static_cast<uint64_t>(n), static_cast<uint64_t>(naux)};
  uint64_t strA[2] = {static_cast<uint64_t>(ldq) * 2, static_cast<uint64_t>(n * ldq) * 2};
  uint32_t boxA[3] = {BK, BM, 1};
  const CUtensorMap a_hi = make_map(mo.bt_hi.p, 3, dimsA, strA, boxA);
  const CUtensorMap a_lo = make_map(mo.bt_lo.p, 3, dimsA, strA, boxA);
  const int bn = rows <= 48 ? 48 : rows <= 80 ? 80 : rows <= 128 ? 128 : rows <= 160 ? 160 : 256;
  RR_REQUIRE(rows >= 1 && rows <= 256, RR_ERR_ARG, "mixed exchange: half-transform pass wider than 256 rows");
  uint64_t dimsB[2] = {static_cast<uint64_t>(n), static_cast<uint64_t>(rows)};
  uint64_t strB[1] = {static_cast<uint64_t>(ldq) * 2};
  uint32_t boxB[2] = {BK, static_cast<uint32_t>(bn)};
  const CUtensorMap b_hi = make_map(coef_hi, 2, dimsB, strB, boxB);
  const CUtensorMap b_lo = make_map(coef_lo, 2, dimsB, strB, boxB);
  const int nkb = static_cast<int>((n + BK - 1) / BK);
  const int mtiles = static_cast<int>((n + BM - 1) / BM);
  const int M = static_cast<int>(n), na = static_cast<int>(naux);
  switch (bn) {
    case 48: return launch_ht_bn<48, 4>(a_hi, a_lo, b_hi, b_lo, e, M, nkb, mtiles, na, err, s);
    case 80: return launch_ht_bn<80, 4>(a_hi, a_lo, b_hi, b_lo, e, M, nkb, mtiles, na, err, s);
    case 128: return launch_ht_bn<128, 3>(a_hi, a_lo, b_hi, b_lo, e, M, nkb, mtiles, na, err, s);
    case 160: return launch_ht_bn<160, 3>(a_hi, a_lo, b_hi, b_lo, e, M, nkb, mtiles, na, err, s);
    default: return launch_ht_bn<256, 2>(a_hi, a_lo, b_hi, b_lo, e, M, nkb, mtiles, na, err, s);
  }
}

// Tile / split layout of one exchange block.
struct BlockPlan {
  int ntm, ntn, tiles, kblocks, splits;
  bool upper;
};

BlockPlan plan_block(int64_t M, int64_t N, int64_t kt, bool upper) {
  BlockPlan b;
  b.ntm = static_cast<int>((M + BM - 1) / BM);
  b.ntn = static_cast<int>((N + GBN - 1) / GBN);
  b.upper = upper;
  b.tiles = upper ? b.ntn * (b.ntn + 1) / 2 : b.ntm * b.ntn;
  b.kblocks = static_cast<int>((kt + BK - 1) / BK);
  int splits = std::max(1, std::min(b.kblocks, static_cast<int>((2LL * sm_count() + b.tiles - 1) / b.tiles)));
  const int per = (b.kblocks + splits - 1) / splits;
  b.splits = (b.kblocks + per - 1) / per;
  return b;
}

// K-contiguous product A (M x kt) . B (N x kt)^T of two split planes (row pitch ldt) into FP32
// partial tiles.
void launch_gemm(const BlockPlan& bp, const uint16_t* a_hi, const uint16_t* a_lo, int64_t M, const uint16_t* b_hi,
                 const uint16_t* b_lo, int64_t N, int64_t kt, int64_t ldt, float* work, int* err, cudaStream_t s) {
  uint64_t dimsA[2] = {static_cast<uint64_t>(kt), static_cast<uint64_t>(M)};
  uint64_t dimsB[2] = {static_cast<uint64_t>(kt), static_cast<uint64_t>(N)};
  uint64_t str[1] = {static_cast<uint64_t>(ldt) * 2};
  uint32_t boxA[2] = {BK, BM};
  uint32_t boxB[2] = {BK, GBN};
  const CUtensorMap mah = make_map(a_hi, 2, dimsA, str, boxA);
  const CUtensorMap mal = make_map(a_lo, 2, dimsA, str, boxA);
  const CUtensorMap mbh = make_map(b_hi, 2, dimsB, str, boxB);
  const CUtensorMap mbl = make_map(b_lo, 2, dimsB, str, boxB);
  GParams p{};
  p.kblocks = bp.kblocks;
  p.splits = bp.splits;
  p.tiles = bp.tiles;
  p.ntn = bp.ntn;
  p.upper = bp.upper ? 1 : 0;
  p.work = work;
  p.err = err;
  static std::atomic<bool> attr[kMaxDevices];
  once_per_device(attr, [] {
    RR_CUDA(cudaFuncSetAttribute(umma_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, GCfg::SMEM));
  });
  umma_gemm_kernel<<<dim3(static_cast<unsigned>(bp.tiles), static_cast<unsigned>(bp.splits)), 128, GCfg::SMEM, s>>>(
      mah, mal, mbh, mbl, p);
  RR_LAUNCH_CHECK();
}

}  // namespace

CUtensorMap bf16_tensor_map(const void* base, int rank, const uint64_t* dims, const uint64_t* strides_bytes,
                            const uint32_t* box, int swizzle_bytes) {
  RR_REQUIRE(swizzle_bytes == 128 || swizzle_bytes == 64, RR_ERR_ARG, "bf16_tensor_map: swizzle of 128 or 64 bytes");
  if (swizzle_bytes == 128) return make_map(base, rank, dims, strides_bytes, box);
  CUtensorMap m;
  uint32_t elem[3] = {1, 1, 1};
  const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, static_cast<cuuint32_t>(rank), const_cast<void*>(base),
                                 reinterpret_cast<const cuuint64_t*>(dims), reinterpret_cast<const cuuint64_t*>(strides_bytes),
                                 reinterpret_cast<const cuuint32_t*>(box), reinterpret_cast<const cuuint32_t*>(elem),
                                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  RR_REQUIRE(r == CUDA_SUCCESS, RR_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(static_cast<int>(r)) + ")");
  return m;
}

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

void mixed_exchange_general(const MixedOperands* ops, MixedScratch& scr, const ExFlavours& fl, int64_t naux,
                            const double* Ct, const double* Ct_prev, int64_t ld, int64_t r, bool cplx, double* K,
                            int64_t ldk, bool accumulate, int* err, cudaStream_t s) {
  RR_REQUIRE(fl.nf >= 1 && fl.nf <= 4, RR_ERR_ARG, "mixed exchange: 1 to 4 flavour blocks");
  RR_REQUIRE(cplx || fl.nf == 1, RR_ERR_ARG, "mixed exchange: real coefficients need a single flavour");
  RR_REQUIRE(naux <= 65535, RR_ERR_ARG, "mixed exchange: naux exceeds the grid limits");
  for (int f = 0; f < fl.nf; ++f) {
    const MixedOperands& mo = ops[fl.tens[f]];
    RR_REQUIRE(mo.ready && mo.n == fl.fs[f] && mo.naux == naux, RR_ERR_STATE, "mixed exchange: operands not prepared");
    RR_REQUIRE(fl.fs[f] <= 65535, RR_ERR_ARG, "mixed exchange: dimensions exceed the grid limits");
  }
  const int pl = cplx ? 2 : 1;
  if (!accumulate) RR_CUDA(cudaMemsetAsync(K, 0, sizeof(double) * ldk * ldk * pl, s));
  if (r == 0 || naux == 0) return;
  // Full build:        coefficient rows [Ct] (real) or [Re Ct, Im Ct]; planes A = T, (complex) B_im =
  //                    [Im, -Re]; blocks f <= u: Re K = A_f A_u^T (Hermitian diagonal blocks: upper
  //                    tiles), Im K = A_f B_im,u^T.
  // Incremental build: rows [W, U] or [Re W, Im W, Re U, Im U]; planes A = W part, B_re = U part,
  //                    (complex) B_im = [Im U, -Re U]; X_fu = A_f B_u^T for every ordered pair (f, u),
  //                    then K += X + X^dagger (= K(Ct) - K(Ct_prev)).
  const bool incr = Ct_prev != nullptr;
  const int mode = cplx ? (incr ? 3 : 2) : (incr ? 1 : 0);
  const int nblk = mode == 0 ? 1 : (mode == 3 ? 4 : 2);      // coefficient blocks per flavour group
  const int oblk = incr ? nblk / 2 : nblk;                     // blocks per aux index in a plane
  const int planes = mode == 0 ? 1 : (mode == 3 ? 3 : 2);
  const int pre = incr ? 1 : 0;  // plane holding the B operand of the real part (imaginary: the last plane)
  // Occupied rows per slice: one flavour's group must fit a 256-column accumulator.
  const int64_t rs_max = 256 / nblk;
  const int64_t nslices = (r + rs_max - 1) / rs_max;
  const int64_t rs_full = (r + nslices - 1) / nslices;
  const int r8 = static_cast<int>(round8(rs_full));
  const int period = nblk * r8, operiod = oblk * r8;
  const int64_t kt = naux * operiod, ldt = round8(kt);
  // Passes: flavours of one tensor, two per pass when both groups fit 256 columns.
  int ntens = 1;
  for (int f = 0; f < fl.nf; ++f) ntens = std::max(ntens, fl.tens[f] + 1);
  struct Pass { int t, g, f0, f1; };
  std::vector<Pass> passes;
  for (int t = 0; t < ntens; ++t) {
    std::vector<int> fs_of;
    for (int f = 0; f < fl.nf; ++f)
      if (fl.tens[f] == t) fs_of.push_back(f);
    const bool two = 2 * period <= 256;
    for (size_t i = 0; i < fs_of.size();) {
      if (two && i + 1 < fs_of.size()) {
        passes.push_back({t, 2, fs_of[i], fs_of[i + 1]});
        i += 2;
      } else {
        passes.push_back({t, 1, fs_of[i], fs_of[i]});
        i += 1;
      }
    }
  }
  // Exchange products of one slice: (f, u, upper tiles).
  struct Blk { int f, u; bool upper; };
  std::vector<Blk> blocks;
  for (int f = 0; f < fl.nf; ++f)
    for (int u = 0; u < fl.nf; ++u) {
      if (!incr && u < f) continue;
      blocks.push_back({f, u, !incr && f == u});
    }
  // Scratch sizes for the whole call, before the first launch.
  int64_t coef_sz = 0, pl_sz = 0, work_sz = 0;
  int64_t pl_off[4];
  for (const Pass& p : passes) coef_sz = std::max<int64_t>(coef_sz, static_cast<int64_t>(p.g) * period * ops[p.t].ldq);
  for (int f = 0; f < fl.nf; ++f) {
    pl_off[f] = pl_sz;
    pl_sz += round_up(planes * fl.fs[f] * ldt, 128);
  }
  for (const Blk& b : blocks) {
    const BlockPlan bp = plan_block(fl.fs[b.f], fl.fs[b.u], kt, b.upper);
    work_sz = std::max<int64_t>(work_sz, pl * static_cast<int64_t>(bp.splits) * bp.tiles * BM * GBN);
  }
  scr.coef_hi.ensure(static_cast<size_t>(coef_sz));
  scr.coef_lo.ensure(static_cast<size_t>(coef_sz));
  scr.pl_hi.ensure(static_cast<size_t>(pl_sz));
  scr.pl_lo.ensure(static_cast<size_t>(pl_sz));
  scr.work.ensure(static_cast<size_t>(work_sz));
  if (incr) scr.xacc.ensure(static_cast<size_t>(ldk * ldk * pl));
  double* target = incr ? scr.xacc.p : K;  // X (incremental) or K itself
  if (incr) RR_CUDA(cudaMemsetAsync(target, 0, sizeof(double) * ldk * ldk * pl, s));
  auto plane = [&](uint16_t* base, int f, int o) { return base + pl_off[f] + static_cast<int64_t>(o) * fl.fs[f] * ldt; };

  // Plane layouts per mode: destination block (-1: not in this plane) and sign of each source block.
  signed char dst[3][4] = {{0, 1, 2, 3}, {-1, -1, -1, -1}, {-1, -1, -1, -1}};
  signed char sgn[3][4] = {{1, 1, 1, 1}, {1, 1, 1, 1}, {1, 1, 1, 1}};
  if (mode == 1) {  // [W, U]: A = W, B = U
    dst[0][1] = -1;
    dst[1][1] = 0;
  } else if (mode == 2) {  // [Re, Im]: A = [Re, Im], B_im = [Im, -Re]
    dst[1][0] = 1; dst[1][1] = 0;
    sgn[1][0] = -1;
  } else if (mode == 3) {  // [Wr, Wi, Ur, Ui]: A = [Wr, Wi], B_re = [Ur, Ui], B_im = [Ui, -Ur]
    dst[0][2] = -1; dst[0][3] = -1;
    dst[1][2] = 0; dst[1][3] = 1;
    dst[2][2] = 1; dst[2][3] = 0;
    sgn[2][2] = -1;
  }

  for (int64_t sl = 0; sl < nslices; ++sl) {
    const int64_t i0 = sl * rs_full;
    const int rs = static_cast<int>(std::min<int64_t>(rs_full, r - i0));
    for (const Pass& p : passes) {
      const MixedOperands& mo = ops[p.t];
      const int rows = p.g * period;
      coef_rows_kernel<<<grid_for(static_cast<int64_t>(rows) * mo.n), 256, 0, s>>>(
          Ct, Ct_prev, ld, i0, rs, r8, mode, p.g, fl.off[p.f0], fl.off[p.f1], static_cast<int>(mo.n),
          static_cast<int>(mo.ldq), reinterpret_cast<__nv_bfloat16*>(scr.coef_hi.p),
          reinterpret_cast<__nv_bfloat16*>(scr.coef_lo.p));
      RR_LAUNCH_CHECK();
      HtEpi e{};
      for (int g = 0; g < p.g; ++g) {
        const int f = g == 0 ? p.f0 : p.f1;
        for (int o = 0; o < planes; ++o) {
          e.hi[g][o] = reinterpret_cast<__nv_bfloat16*>(plane(scr.pl_hi.p, f, o));
          e.lo[g][o] = reinterpret_cast<__nv_bfloat16*>(plane(scr.pl_lo.p, f, o));
        }
      }
      e.ld = ldt;
      e.ncols = rows;
      e.groups = p.g;
      e.planes = planes;
      e.period = period;
      e.operiod = operiod;
      e.blk = r8;
      std::memcpy(e.dst, dst, sizeof(dst));
      std::memcpy(e.sgn, sgn, sizeof(sgn));
      launch_ht(mo, scr.coef_hi.p, scr.coef_lo.p, rows, e, err, s);
    }
    for (const Blk& b : blocks) {
      const BlockPlan bp = plan_block(fl.fs[b.f], fl.fs[b.u], kt, b.upper);
      const int64_t part = static_cast<int64_t>(bp.splits) * bp.tiles * BM * GBN;
      float* wre = scr.work.p;
      float* wim = cplx ? scr.work.p + part : nullptr;
      launch_gemm(bp, plane(scr.pl_hi.p, b.f, 0), plane(scr.pl_lo.p, b.f, 0), fl.fs[b.f], plane(scr.pl_hi.p, b.u, pre),
                  plane(scr.pl_lo.p, b.u, pre), fl.fs[b.u], kt, ldt, wre, err, s);
      if (cplx)
        launch_gemm(bp, plane(scr.pl_hi.p, b.f, 0), plane(scr.pl_lo.p, b.f, 0), fl.fs[b.f],
                    plane(scr.pl_hi.p, b.u, planes - 1), plane(scr.pl_lo.p, b.u, planes - 1), fl.fs[b.u], kt, ldt,
                    wim, err, s);
      const int both = !incr && b.f != b.u ? 1 : 0;
      umma_place_kernel<<<grid_for(fl.fs[b.f] * fl.fs[b.u]), 256, 0, s>>>(
          wre, wim, bp.splits, bp.tiles, bp.ntn, bp.upper ? 1 : 0, static_cast<int>(fl.fs[b.f]),
          static_cast<int>(fl.fs[b.u]), target, ldk, fl.off[b.f], fl.off[b.u], both, 1, cplx ? 1 : 0);
      RR_LAUNCH_CHECK();
    }
  }
  if (incr) {
    herm_add_kernel<<<grid_for(ldk * ldk), 256, 0, s>>>(K, scr.xacc.p, ldk, 1, cplx ? 1 : 0);
    RR_LAUNCH_CHECK();
  }
}

void mixed_exchange(const MixedOperands& mo, MixedScratch& scr, const double* Ct, int64_t ldct, int64_t nocc, double* K,
                    int* err, cudaStream_t s) {
  ExFlavours fl;
  fl.nf = 1;
  fl.fs[0] = mo.n;
  mixed_exchange_general(&mo, scr, fl, mo.naux, Ct, nullptr, ldct, nocc, false, K, mo.n, false, err, s);
}

}  // namespace rr
