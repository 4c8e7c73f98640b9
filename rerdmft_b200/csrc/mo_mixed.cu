// Split-BF16 MO three-index transforms on the 5th-generation tensor cores (RR_PREC_MIXED of
// rr_mo_build_nonrel and rr_mo_build_ukb).  Nonrelativistic: B_mo^P = C^T B^P C for every aux index P; the
// complex four-block form (buildRiMoEri) reuses the same kernel with other operand rows and output maps
// (mo_build_ukb_mixed below).
//
// The reference forms the two products per P in FP64 (src/NON_REL/NonRelSpinRiMoEri.cpp:13-43,
// buildRiNonRelSpinMoEri).  Here both products run as split-BF16 tcgen05 MMAs (x y ~= hi hi + hi lo +
// lo hi, FP32 accumulation in TMEM), each as ONE flat GEMM over all aux indices, K-contiguous operands
// staged by TMA:
//   step 1  Y[(P, a)][j] = sum_q Bt[P][a][q] Ct[j][q]        (= (B^P^T C)[a][j])
//           rows (P, a) of the resident split copy of B, columns j of Ct = C^T (the same 128-row tile of
//           B serves every column tile); the epilogue writes Y transposed and split, Yt[P][j][a];
//   step 2  O[(P, j)][i] = sum_a Yt[P][j][a] Ct[i][a]         (= (C^T B^P C)[j][i])
//           rows (P, j) of Yt, the same Ct operand; the epilogue writes O in FP64 straight into the
//           resident MO tensor, B_mo[P][j][i].
// Neither step needs symmetry of B^P: the result is C^T B^P C element for element.
// Kernel: one persistent CTA per SM walks (row tile, column tile) items with a continuous TMA ring and
// two TMEM accumulators, so the epilogue of one item overlaps the MMAs of the next.  Roles: warps 0-3
// drain TMEM (lanes 32 w .. 32 w + 31) through a per-warp shared-memory staging tile, so that the stores
// are whole 16-byte BF16 runs or whole FP64 row segments; warp 4 lane 0 issues the TMA ring, warp 5 lane 0
// the MMAs.
// Every mbarrier wait is bounded; an expiry sets a status bit that the host reports as RR_ERR_TIMEOUT.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>

#include "mixed.cuh"
#include "mo_store.cuh"
#include "ri_store.cuh"
#include "umma.cuh"

namespace rr {

namespace {

constexpr int BM = 128;
// K blocks: SWZ = 128 (64 BF16 per 128-byte swizzled row) or SWZ = 64 (32 BF16 per 64-byte row: half the
// bytes per ring stage, so twice the stages in flight, and K padded to 32 instead of 64).
template <int SWZ>
struct KBlk {
  static constexpr int BK = SWZ / 2;
  static constexpr int A_TILE = BM * BK * 2;  // bytes
};
constexpr int MO_THREADS = 192;
constexpr int ERR_MO_FULL = 1 << 12, ERR_MO_EMPTY = 1 << 13, ERR_MO_TFULL = 1 << 14, ERR_MO_TEMPTY = 1 << 15,
              ERR_MO_DONE = 1 << 16;

template <int BN, int STAGES, int SWZ>
struct MoCfg {
  static constexpr int BK = KBlk<SWZ>::BK;
  static constexpr int A_TILE = KBlk<SWZ>::A_TILE;
  static constexpr int B_TILE = BN * BK * 2;
  static constexpr int STAGE = 2 * A_TILE + 2 * B_TILE;
  static constexpr int BNP = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));  // TMEM columns per accumulator
  static constexpr int TMEM_COLS = 2 * BNP <= 64 ? 64 : (2 * BNP <= 128 ? 128 : (2 * BNP <= 256 ? 256 : 512));
  static constexpr int EPI_OFF = STAGES * STAGE + 256;        // epilogue staging: 4 warps x 32 x 33 floats
  static constexpr int SMEM = EPI_OFF + 4 * 32 * 33 * 4 + 1024;
  static_assert(B_TILE % (8 * SWZ) == 0 && A_TILE % (8 * SWZ) == 0, "tiles keep the swizzle-atom alignment");
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "UMMA N for M = 128");
  static_assert(SMEM <= 232448, "shared memory per CTA");
};

// Output of one step.  Row R of the flat product is (P, r) with P = R / rper, r = R % rper; column c < ncol.
//   EPI 0: hi/lo[(P cmod + c % cmod) ldq + (c / cmod) chi + koff + r] = split(value), ncol <= 2 cmod
//          (nonrelativistic: cmod = n, Yt[P][c][r]; complex: c = (Re | Im block, q), K index of r shifted by
//          the flavour's UKB row offset koff and by chi = n_ukb for the imaginary block)
//   EPI 1: out[R ldo + c] = value, negated for odd c when conj_odd (the imaginary parts of a conjugate)
struct MoEpi {
  int64_t rows;
  int rper, ncol, cmod;
  int64_t chi, koff, ldq;
  __nv_bfloat16* hi;
  __nv_bfloat16* lo;
  int64_t ldo;
  int conj_odd;
  double* out;
};

__device__ __forceinline__ uint32_t pack2_bf16(float x, float y) {
  return static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16_rn(x))) |
         (static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16_rn(y))) << 16);
}

// 32 lanes x 32 columns of 32-bit TMEM data per warp, load and wait in one statement.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
      "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// K-major shared-memory descriptor for a 64-byte swizzle: 8-row atoms of 512 bytes (stride byte offset 512),
// leading byte offset unused (1), descriptor version 1, layout type 4 (64-byte swizzle).
__device__ __forceinline__ uint64_t sdesc_k_sw64(uint32_t smem_addr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((smem_addr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>(1u) << 16;
  d |= static_cast<uint64_t>(512u >> 4) << 32;
  d |= static_cast<uint64_t>(1u) << 46;
  d |= static_cast<uint64_t>(4u) << 61;
  return d;
}

template <int SWZ>
__device__ __forceinline__ uint64_t sdesc_k(uint32_t smem_addr) {
  return SWZ == 128 ? sdesc_k_sw128(smem_addr) : sdesc_k_sw64(smem_addr);
}

template <int BN, int STAGES, int EPI, int SWZ>
__global__ void __launch_bounds__(MO_THREADS, 1)
    umma_mo_kernel(const __grid_constant__ CUtensorMap mapA_hi, const __grid_constant__ CUtensorMap mapA_lo,
                   const __grid_constant__ CUtensorMap mapB_hi, const __grid_constant__ CUtensorMap mapB_lo,
                   const MoEpi e, int nkb, int kvalid, int64_t rtiles, int ntn, int* err) {
  using CF = MoCfg<BN, STAGES, SWZ>;
  constexpr int BK = CF::BK, A_TILE = CF::A_TILE;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * CF::STAGE);
  uint64_t* empty = full + STAGES;
  uint64_t* tfull = empty + STAGES;
  uint64_t* tempty = tfull + 2;
  uint64_t* mdone = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mdone + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t total = rtiles * ntn;

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
    if (lane == 0) {  // TMA producer; column tiles of one row tile are consecutive items (A tile reuse in L2)
      uint32_t q = 0;
      for (int64_t item = blockIdx.x; item < total && !dead; item += gridDim.x) {
        const int r0 = static_cast<int>((item / ntn) * BM), n0 = static_cast<int>(item % ntn) * BN;
        for (int k = 0; k < nkb; ++k, ++q) {
          const int s = q % STAGES;
          if (q >= STAGES && !mbar_wait(&empty[s], ((q / STAGES) & 1) ^ 1, err, ERR_MO_EMPTY, dead)) break;
          unsigned char* st = smem + s * CF::STAGE;
          const int kc = k * BK;
          mbar_arrive_expect_tx(&full[s], CF::STAGE);
          tma_load_2d(st, &mapA_hi, kc, r0, &full[s]);
          tma_load_2d(st + A_TILE, &mapA_lo, kc, r0, &full[s]);
          tma_load_2d(st + 2 * A_TILE, &mapB_hi, kc, n0, &full[s]);
          tma_load_2d(st + 2 * A_TILE + CF::B_TILE, &mapB_lo, kc, n0, &full[s]);
        }
      }
    }
  } else if (warp == 5) {
    if (lane == 0) {  // MMA issuer
      uint32_t q = 0, j = 0;
      for (int64_t item = blockIdx.x; item < total; item += gridDim.x, ++j) {
        const uint32_t b = j & 1;
        // the last column tile multiplies only its valid columns (rounded up to the UMMA N step of 16)
        const int nv = min(BN, e.ncol - static_cast<int>(item % ntn) * BN);
        const uint32_t idesc = idesc_bf16_f32(BM, (nv + 15) / 16 * 16);
        if (j >= 2) mbar_wait(&tempty[b], ((j >> 1) - 1) & 1, err, ERR_MO_TEMPTY, dead);
        tc_fence_after();
        const uint32_t d = tmem + b * CF::BNP;
        for (int k = 0; k < nkb; ++k, ++q) {
          const int s = q % STAGES;
          mbar_wait(&full[s], (q / STAGES) & 1, err, ERR_MO_FULL, dead);
          tc_fence_after();
          if (!dead) {
            const uint32_t base = smem_u32(smem + s * CF::STAGE);
            const uint64_t ahi = sdesc_k<SWZ>(base), alo = sdesc_k<SWZ>(base + A_TILE);
            const uint64_t bhi = sdesc_k<SWZ>(base + 2 * A_TILE), blo = sdesc_k<SWZ>(base + 2 * A_TILE + CF::B_TILE);
            const int nks = min(BK / 16, (kvalid - k * BK + 15) / 16);  // 16-deep steps holding data (zero fill beyond)
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
              if (kk >= nks) break;
              const uint64_t dk = static_cast<uint64_t>(kk * 32) >> 4;  // +32 bytes per 16-element step
              umma_bf16(d, ahi + dk, bhi + dk, idesc, (k > 0 || kk > 0) ? 1u : 0u);
              umma_bf16(d, ahi + dk, blo + dk, idesc, 1u);
              umma_bf16(d, alo + dk, bhi + dk, idesc, 1u);
            }
          }
          umma_commit(&empty[s]);  // frees the stage once these MMAs have read it
        }
        umma_commit(&tfull[b]);
        if (dead) break;
      }
      umma_commit(mdone);
    }
  } else {  // epilogue warps 0-3
    uint32_t j = 0;
    const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
    float* sw = reinterpret_cast<float*>(smem + CF::EPI_OFF) + warp * (32 * 33);  // this warp's 32 x 32 staging tile
    for (int64_t item = blockIdx.x; item < total; item += gridDim.x, ++j) {
      const uint32_t b = j & 1;
      const bool ok = mbar_wait(&tfull[b], (j >> 1) & 1, err, ERR_MO_TFULL, dead);
      tc_fence_after();
      if (ok) {
        const int64_t R0 = (item / ntn) * BM + warp * 32;  // first row of this warp
        const int64_t R = R0 + lane;
        const int n0 = static_cast<int>(item % ntn) * BN;
        const bool live = R < e.rows;
        const int64_t P = live ? R / e.rper : 0;
        const int r = live ? static_cast<int>(R - P * e.rper) : 0;
        // Fast paths write through the staging tile: EPI 0 as 16-byte runs of 8 consecutive r of one P (all 32
        // rows live and in one P, r 8-aligned), EPI 1 as whole 128- / 256-byte row segments (n even).
        const int64_t P0 = R0 / e.rper;
        const int a0 = static_cast<int>(R0 - P0 * e.rper);
        const bool rows_ok = R0 + 31 < e.rows;
        const bool fast0 = rows_ok && a0 + 31 < e.rper && ((e.koff + a0) & 7) == 0 && (e.chi & 7) == 0 &&
                           (e.ldq & 7) == 0;
        const bool fast1 = rows_ok && (e.ldo & 1) == 0;
        const double sgn_odd = e.conj_odd ? -1.0 : 1.0;
        for (int c0 = 0; c0 < BN && n0 + c0 < e.ncol; c0 += 32) {  // warp-uniform bounds
          const int W = c0 + 32 <= BN ? 32 : 16;                  // BN is a multiple of 16
          float v[32];
          if (W == 32) tmem_ld32(tmem + lane_base + b * CF::BNP + c0, v);
          else tmem_ld16(tmem + lane_base + b * CF::BNP + c0, v);
          const int cb = n0 + c0;
          const int cw = min(W, e.ncol - cb);  // valid columns of this chunk
          __syncwarp();                     // the previous chunk's reads of the tile are done
#pragma unroll
          for (int t = 0; t < 32; ++t)
            if (t < W) sw[lane * 33 + t] = v[t];
          __syncwarp();
          if (EPI == 0) {
            if (fast0) {
              const int g = lane & 3;
              for (int jc = lane >> 2; jc < cw; jc += 8) {
                uint32_t h[4], l[4];
#pragma unroll
                for (int k = 0; k < 8; k += 2) {
                  const float x0 = sw[(8 * g + k) * 33 + jc], x1 = sw[(8 * g + k + 1) * 33 + jc];
                  const float q0 = __bfloat162float(__float2bfloat16_rn(x0)), q1 = __bfloat162float(__float2bfloat16_rn(x1));
                  h[k >> 1] = pack2_bf16(x0, x1);
                  l[k >> 1] = pack2_bf16(x0 - q0, x1 - q1);
                }
                const int col = cb + jc;
                const int blk = col >= e.cmod ? 1 : 0;  // ncol <= 2 cmod
                const int64_t o = (P0 * e.cmod + col - blk * e.cmod) * e.ldq + blk * e.chi + e.koff + a0 + 8 * g;
                *reinterpret_cast<uint4*>(e.hi + o) = make_uint4(h[0], h[1], h[2], h[3]);
                *reinterpret_cast<uint4*>(e.lo + o) = make_uint4(l[0], l[1], l[2], l[3]);
              }
            } else if (live) {
#pragma unroll
              for (int t = 0; t < 32; ++t) {
                if (t >= cw) continue;
                const int col = cb + t;
                const int blk = col >= e.cmod ? 1 : 0;
                const int64_t o = (P * e.cmod + col - blk * e.cmod) * e.ldq + blk * e.chi + e.koff + r;
                const __nv_bfloat16 hb = __float2bfloat16_rn(v[t]);
                e.hi[o] = hb;
                e.lo[o] = __float2bfloat16_rn(v[t] - __bfloat162float(hb));
              }
            }
          } else {
            if (fast1) {
              const int lpr = cw >> 1;  // lanes per row segment (cw even: n even, cb even)
              const int rpi = 32 / W * 2;  // rows per store instruction at a full chunk
              if (cw == W) {
                const int rr0 = lane / lpr, cp = lane % lpr;
                for (int rr = rr0; rr < 32; rr += rpi) {
                  const double2 d = make_double2(static_cast<double>(sw[rr * 33 + 2 * cp]),
                                                 sgn_odd * static_cast<double>(sw[rr * 33 + 2 * cp + 1]));
                  *reinterpret_cast<double2*>(e.out + (R0 + rr) * e.ldo + cb + 2 * cp) = d;
                }
              } else {
#pragma unroll
                for (int t = 0; t < 32; t += 2)
                  if (t < cw)
                    *reinterpret_cast<double2*>(e.out + R * e.ldo + cb + t) =
                        make_double2(static_cast<double>(v[t]), sgn_odd * static_cast<double>(v[t + 1]));
              }
            } else if (live) {
#pragma unroll
              for (int t = 0; t < 32; ++t)
                if (t < cw) e.out[R * e.ldo + cb + t] = (((cb + t) & 1) ? sgn_odd : 1.0) * static_cast<double>(v[t]);
            }
          }
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
    mbar_wait(mdone, 0, err, ERR_MO_DONE, ddead);  // every MMA retired before TMEM is released
    tc_fence_after();
    tmem_dealloc(tmem, CF::TMEM_COLS);
  }
}

// Ct_hi/lo[j][q] (row pitch ldq) = split(C[q][j]) for the n x n row-major C.
__global__ void ct_split_kernel(const double* C, int n, int64_t ldq, __nv_bfloat16* hi, __nv_bfloat16* lo) {
  const int64_t cnt = static_cast<int64_t>(n) * n;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < cnt;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(idx / n), q = static_cast<int>(idx % n);
    const double x = C[static_cast<int64_t>(q) * n + j];
    const __nv_bfloat16 h = __double2bfloat16(x);
    hi[j * ldq + q] = h;
    lo[j * ldq + q] = __double2bfloat16(x - static_cast<double>(__bfloat162float(h)));
  }
}

template <int BN, int STAGES, int EPI, int SWZ>
void launch_mo(const CUtensorMap& a_hi, const CUtensorMap& a_lo, const CUtensorMap& b_hi, const CUtensorMap& b_lo,
               const MoEpi& e, int kvalid, int* err, cudaStream_t s) {
  const int nkb = (kvalid + KBlk<SWZ>::BK - 1) / KBlk<SWZ>::BK;
  using CF = MoCfg<BN, STAGES, SWZ>;
  auto kern = umma_mo_kernel<BN, STAGES, EPI, SWZ>;
  static std::atomic<bool> attr[kMaxDevices];
  once_per_device(attr, [&] { RR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, CF::SMEM)); });
  const int64_t rtiles = (e.rows + BM - 1) / BM;
  const int ntn = (e.ncol + BN - 1) / BN;
  const int64_t items = rtiles * ntn;
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(items, sm_count_current())));
  kern<<<grid, MO_THREADS, CF::SMEM, s>>>(a_hi, a_lo, b_hi, b_lo, e, nkb, kvalid, rtiles, ntn, err);
  RR_LAUNCH_CHECK();
}

// Column tile width: each item streams a 128-row A tile and a BN-row B tile through the ring and issues
// BN-wide MMAs, so cost ~ ntn * (BN + 64) (A weighted half: its rows are shared by the column tiles of a row
// tile in L2).  At n = 400 this orders the tiles as measured: 208 (1.32 ms) < 144 (1.53) < 256 (1.72) < 112
// (1.79) < 128 (1.91 ms per build at naux = 1600).
int pick_bn(int64_t n) {
  const int cand[7] = {32, 64, 112, 128, 144, 208, 256};
  int best = 256;
  int64_t best_cost = (n + 255) / 256 * (256 + 64);
  for (int c : cand) {
    const int64_t cost = (n + c - 1) / c * (c + 64);
    if (cost < best_cost) { best = c; best_cost = cost; }
  }
  return best;
}

template <int EPI>
void launch_step(int bn, int swz, const CUtensorMap& a_hi, const CUtensorMap& a_lo, const CUtensorMap& b_hi,
                 const CUtensorMap& b_lo, const MoEpi& e, int kvalid, int* err, cudaStream_t s) {
  RR_REQUIRE(e.ncol <= 2 * static_cast<int64_t>(e.cmod) && e.rper > 0, RR_ERR_ARG, "MO transform: bad epilogue layout");
  if (swz == 128) {
    switch (bn) {
      case 128: return launch_mo<128, 3, EPI, 128>(a_hi, a_lo, b_hi, b_lo, e, kvalid, err, s);
      case 144: return launch_mo<144, 3, EPI, 128>(a_hi, a_lo, b_hi, b_lo, e, kvalid, err, s);
      default: return launch_mo<208, 2, EPI, 128>(a_hi, a_lo, b_hi, b_lo, e, kvalid, err, s);
    }
  }
  switch (bn) {
    case 32: return launch_mo<32, 8, EPI, 64>(a_hi, a_lo, b_hi, b_lo, e, kvalid, err, s);
    case 64: return launch_mo<64, 8, EPI, 64>(a_hi, a_lo, b_hi, b_lo, e, kvalid, err, s);
    case 112: return launch_mo<112, 6, EPI, 64>(a_hi, a_lo, b_hi, b_lo, e, kvalid, err, s);
    case 128: return launch_mo<128, 6, EPI, 64>(a_hi, a_lo, b_hi, b_lo, e, kvalid, err, s);
    case 144: return launch_mo<144, 6, EPI, 64>(a_hi, a_lo, b_hi, b_lo, e, kvalid, err, s);
    case 208: return launch_mo<208, 4, EPI, 64>(a_hi, a_lo, b_hi, b_lo, e, kvalid, err, s);
    default: return launch_mo<256, 4, EPI, 64>(a_hi, a_lo, b_hi, b_lo, e, kvalid, err, s);
  }
}

// Column tile width and swizzle for a product of `ncol` columns (RR_MO_BN / RR_MO_SWZ force them for
// measurement).  The 128-byte swizzle (64-deep K blocks) where it is instantiated; the 64-byte swizzle's deeper
// ring measured slower at n = 400 (1.371 against 1.321 ms per build with BN = 208).
void choose_tiles(int64_t ncol, int* bn_out, int* swz_out) {
  int bn = pick_bn(ncol);
  if (const char* v = std::getenv("RR_MO_BN")) {
    const int f = std::atoi(v);
    RR_REQUIRE(f == 32 || f == 64 || f == 112 || f == 128 || f == 144 || f == 208 || f == 256, RR_ERR_ARG,
               "RR_MO_BN: one of 32, 64, 112, 128, 144, 208, 256");
    bn = f;
  }
  int swz = (bn == 128 || bn == 144 || bn == 208) ? 128 : 64;
  if (const char* v = std::getenv("RR_MO_SWZ")) {
    swz = std::atoi(v);
    RR_REQUIRE((swz == 64) || (swz == 128 && (bn == 128 || bn == 144 || bn == 208)), RR_ERR_ARG,
               "RR_MO_SWZ: 64, or 128 with a column tile of 128, 144 or 208");
  }
  *bn_out = bn;
  *swz_out = swz;
}

// Split rows of the complex transform's B operands (BF16 hi / lo, row pitch ld) from c (nu x nt complex,
// interleaved, row-major):
//   ct2 of a flavour block (rows [off, off + fs) of c):  ct2[j'][q] = Re c[off + q][j'] (j' < nt),
//                                                         Im c[off + q][j' - nt] (j' >= nt);
//   cc over all rows k of c (K = 2 nu):  cc[2p][k] = Re c[k][p], cc[2p][nu + k] = Im c[k][p],
//                                         cc[2p + 1][k] = -Im c[k][p], cc[2p + 1][nu + k] = Re c[k][p].
__global__ void ct2_split_kernel(const double* c, int64_t nt, int64_t off, int64_t fs, int64_t ld, __nv_bfloat16* hi,
                                 __nv_bfloat16* lo) {
  const int64_t cnt = 2 * nt * fs;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < cnt;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t jp = idx / fs, q = idx % fs;
    const int part = jp >= nt ? 1 : 0;
    const double x = c[((off + q) * nt + (jp - part * nt)) * 2 + part];
    const __nv_bfloat16 h = __double2bfloat16(x);
    hi[jp * ld + q] = h;
    lo[jp * ld + q] = __double2bfloat16(x - static_cast<double>(__bfloat162float(h)));
  }
}

__global__ void cc_split_kernel(const double* c, int64_t nt, int64_t nu, int64_t ld, __nv_bfloat16* hi,
                                __nv_bfloat16* lo) {
  const int64_t cnt = 2 * nt * 2 * nu;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < cnt;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t row = idx / (2 * nu), k = idx % (2 * nu);
    const int64_t p = row >> 1;
    const bool second = k >= nu;
    const double* e = c + ((second ? k - nu : k) * nt + p) * 2;
    const double x = (row & 1) ? (second ? e[0] : -e[1]) : (second ? e[1] : e[0]);
    const __nv_bfloat16 h = __double2bfloat16(x);
    hi[row * ld + k] = h;
    lo[row * ld + k] = __double2bfloat16(x - static_cast<double>(__bfloat162float(h)));
  }
}

int grid_of(int64_t count) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((count + 255) / 256, 1184))); }

}  // namespace

void mo_build_nonrel_mixed(rr_ri_store* ri, const double* C, rr_mo_store* m, bool host, cudaStream_t s) {
  const int64_t n = ri->n, naux = ri->naux;
  RR_REQUIRE(n <= 65535 && naux * n < (int64_t(1) << 31), RR_ERR_ARG,
             "rr_mo_build_nonrel (RR_PREC_MIXED): naux * n exceeds the tensor-map limits");
  m->B.ensure(static_cast<size_t>(std::max<int64_t>(naux * n * n, 1)));  // a rebuild keeps the tensor's memory
  if (n == 0 || naux == 0) return;
  m->scratch.ensure(static_cast<size_t>(round_up(n * n, 32)));
  double* Cd = m->scratch.p;
  copy_in(Cd, C, n * n, host, s);
  mixed_prepare(ri->mixed[0], ri->B[0].p, ri->pitch[0], n, naux, s);
  const MixedOperands& mo = ri->mixed[0];
  const int64_t ldq = mo.ldq;
  MixedScratch& scr = ri->mscr;
  scr.coef_hi.ensure(static_cast<size_t>(n * ldq));
  scr.coef_lo.ensure(static_cast<size_t>(n * ldq));
  scr.pl_hi.ensure(static_cast<size_t>(naux * n * ldq));
  scr.pl_lo.ensure(static_cast<size_t>(naux * n * ldq));
  auto* ct_hi = reinterpret_cast<__nv_bfloat16*>(scr.coef_hi.p);
  auto* ct_lo = reinterpret_cast<__nv_bfloat16*>(scr.coef_lo.p);
  ct_split_kernel<<<static_cast<int>(std::min<int64_t>((n * n + 255) / 256, 1184)), 256, 0, s>>>(Cd, static_cast<int>(n),
                                                                                                 ldq, ct_hi, ct_lo);
  RR_LAUNCH_CHECK();

  int bn = 0, swz = 0;
  choose_tiles(n, &bn, &swz);
  const int BK = swz / 2;
  const uint64_t rows = static_cast<uint64_t>(naux * n);
  uint64_t dimsA[2] = {static_cast<uint64_t>(n), rows};
  uint64_t dimsB[2] = {static_cast<uint64_t>(n), static_cast<uint64_t>(n)};
  uint64_t str[1] = {static_cast<uint64_t>(ldq) * 2};
  uint32_t boxA[2] = {static_cast<uint32_t>(BK), BM};
  uint32_t boxB[2] = {static_cast<uint32_t>(BK), static_cast<uint32_t>(bn)};
  const CUtensorMap bt_hi = bf16_tensor_map(mo.bt_hi.p, 2, dimsA, str, boxA, swz);
  const CUtensorMap bt_lo = bf16_tensor_map(mo.bt_lo.p, 2, dimsA, str, boxA, swz);
  const CUtensorMap c_hi = bf16_tensor_map(ct_hi, 2, dimsB, str, boxB, swz);
  const CUtensorMap c_lo = bf16_tensor_map(ct_lo, 2, dimsB, str, boxB, swz);
  const CUtensorMap y_hi = bf16_tensor_map(scr.pl_hi.p, 2, dimsA, str, boxA, swz);
  const CUtensorMap y_lo = bf16_tensor_map(scr.pl_lo.p, 2, dimsA, str, boxA, swz);

  MoEpi e{};
  e.rows = naux * n;
  e.rper = e.ncol = e.cmod = static_cast<int>(n);
  e.chi = 0;
  e.koff = 0;
  e.ldq = ldq;
  e.hi = reinterpret_cast<__nv_bfloat16*>(scr.pl_hi.p);
  e.lo = reinterpret_cast<__nv_bfloat16*>(scr.pl_lo.p);
  e.ldo = n;
  e.conj_odd = 0;
  e.out = m->B.p;
  launch_step<0>(bn, swz, bt_hi, bt_lo, c_hi, c_lo, e, static_cast<int>(n), ri->status.p, s);  // Yt = (B^P^T C)^T, split
  launch_step<1>(bn, swz, y_hi, y_lo, c_hi, c_lo, e, static_cast<int>(n), ri->status.p, s);    // B_mo^P = C^T B^P C
}

// RR_PREC_MIXED buildRiMoEri (src/UKB/RiMoEri.cpp:20-86): B(P,p,q) = sum_f c_f^dagger B_f^P c_f over the four
// UKB blocks, c = R + i I.  Step 1 per flavour f: Y_f = B_f^T [R_f | I_f] (real, 2 nt columns) written as
// Yt[P][q][k] with k = off_f + a for the real block and nu + off_f + a for the imaginary one, so every flavour
// lands in one K range of length 2 nu.  Step 2, one real GEMM with K = 2 nu over all flavours:
//   M[p][q] = sum_f c_f^dagger (B_f^T c_f) = sum_k cc[2p][k] Yt[q][k] + i sum_k cc[2p + 1][k] Yt[q][k]
// with the output row (P, q) and the interleaved column (p, Re / Im): stored as B[P][q][p] = conj(M[p][q]),
// which is (c^dagger B c)[q][p] element for element (no symmetry of B_f^P needed).  Chunked over P so that
// the split intermediate stays within 256 Mi elements a plane.
void mo_build_ukb_mixed(rr_ri_store* ri, const double* c_ukb, int64_t nt, rr_mo_store* m, bool host, cudaStream_t s) {
  const int64_t nl = ri->n, ns = ri->ns, naux = ri->naux, nu = 2 * nl + 2 * ns;
  const int64_t off[4] = {0, nl, 2 * nl, 2 * nl + ns}, fs[4] = {nl, nl, ns, ns};
  const int tens[4] = {0, 0, 1, 1};
  const int64_t fsmax = std::max(nl, ns);
  RR_REQUIRE(2 * nt <= 65535 && fsmax <= 65535 && naux * std::max(fsmax, nt) < (int64_t(1) << 31), RR_ERR_ARG,
             "rr_mo_build_ukb (RR_PREC_MIXED): dimensions exceed the tensor-map limits");
  m->B.ensure(static_cast<size_t>(std::max<int64_t>(2 * naux * nt * nt, 1)));
  if (nt == 0 || naux == 0 || nu == 0) {
    if (m->B.n) RR_CUDA(cudaMemsetAsync(m->B.p, 0, sizeof(double) * m->B.n, s));
    return;
  }
  m->scratch.ensure(static_cast<size_t>(round_up(2 * nu * nt, 32)));
  double* cd = m->scratch.p;
  copy_in(cd, c_ukb, 2 * nu * nt, host, s);
  for (int t = 0; t < 2; ++t) {
    const int64_t ft = t == 0 ? nl : ns;
    if (ft > 0) mixed_prepare(ri->mixed[t], ri->B[t].p, ri->pitch[t], ft, naux, s);
  }
  const int64_t K2 = 2 * nu, ldk = (K2 + 7) / 8 * 8;
  // B operands: cc (2 nt x ldk) and one ct2 per flavour (2 nt x ldq of its tensor), 256-element aligned
  int64_t ooff[5];
  int64_t tot = round_up(2 * nt * ldk, 256);
  for (int f = 0; f < 4; ++f) {
    ooff[f] = tot;
    tot += fs[f] > 0 ? round_up(2 * nt * ri->mixed[tens[f]].ldq, 256) : 0;
  }
  MixedScratch& scr = ri->mscr;
  scr.coef_hi.ensure(static_cast<size_t>(tot));
  scr.coef_lo.ensure(static_cast<size_t>(tot));
  auto* ch = reinterpret_cast<__nv_bfloat16*>(scr.coef_hi.p);
  auto* cl = reinterpret_cast<__nv_bfloat16*>(scr.coef_lo.p);
  cc_split_kernel<<<grid_of(2 * nt * K2), 256, 0, s>>>(cd, nt, nu, ldk, ch, cl);
  RR_LAUNCH_CHECK();
  for (int f = 0; f < 4; ++f) {
    if (fs[f] == 0) continue;
    ct2_split_kernel<<<grid_of(2 * nt * fs[f]), 256, 0, s>>>(cd, nt, off[f], fs[f], ri->mixed[tens[f]].ldq, ch + ooff[f],
                                                             cl + ooff[f]);
    RR_LAUNCH_CHECK();
  }
  const int64_t pc = std::max<int64_t>(1, std::min<int64_t>(naux, (int64_t(1) << 28) / (nt * ldk)));
  scr.pl_hi.ensure(static_cast<size_t>(pc * nt * ldk));
  scr.pl_lo.ensure(static_cast<size_t>(pc * nt * ldk));
  int bn = 0, swz = 0;
  choose_tiles(2 * nt, &bn, &swz);
  const int BK = swz / 2;
  uint32_t boxA[2] = {static_cast<uint32_t>(BK), BM};
  uint32_t boxB[2] = {static_cast<uint32_t>(BK), static_cast<uint32_t>(bn)};
  uint64_t strk[1] = {static_cast<uint64_t>(ldk) * 2};
  uint64_t dimsC[2] = {static_cast<uint64_t>(K2), static_cast<uint64_t>(2 * nt)};
  const CUtensorMap cc_hi = bf16_tensor_map(ch, 2, dimsC, strk, boxB, swz);
  const CUtensorMap cc_lo = bf16_tensor_map(cl, 2, dimsC, strk, boxB, swz);
  for (int64_t P0 = 0; P0 < naux; P0 += pc) {
    const int64_t cnt = std::min(pc, naux - P0);
    for (int f = 0; f < 4; ++f) {  // step 1: Yt columns of flavour f
      if (fs[f] == 0) continue;
      const MixedOperands& mo = ri->mixed[tens[f]];
      uint64_t dimsA[2] = {static_cast<uint64_t>(fs[f]), static_cast<uint64_t>(cnt * fs[f])};
      uint64_t dimsB[2] = {static_cast<uint64_t>(fs[f]), static_cast<uint64_t>(2 * nt)};
      uint64_t strq[1] = {static_cast<uint64_t>(mo.ldq) * 2};
      const int64_t a_off = P0 * fs[f] * mo.ldq;
      const CUtensorMap a_hi = bf16_tensor_map(mo.bt_hi.p + a_off, 2, dimsA, strq, boxA, swz);
      const CUtensorMap a_lo = bf16_tensor_map(mo.bt_lo.p + a_off, 2, dimsA, strq, boxA, swz);
      const CUtensorMap b_hi = bf16_tensor_map(ch + ooff[f], 2, dimsB, strq, boxB, swz);
      const CUtensorMap b_lo = bf16_tensor_map(cl + ooff[f], 2, dimsB, strq, boxB, swz);
      MoEpi e{};
      e.rows = cnt * fs[f];
      e.rper = static_cast<int>(fs[f]);
      e.ncol = static_cast<int>(2 * nt);
      e.cmod = static_cast<int>(nt);
      e.chi = nu;
      e.koff = off[f];
      e.ldq = ldk;
      e.hi = reinterpret_cast<__nv_bfloat16*>(scr.pl_hi.p);
      e.lo = reinterpret_cast<__nv_bfloat16*>(scr.pl_lo.p);
      launch_step<0>(bn, swz, a_hi, a_lo, b_hi, b_lo, e, static_cast<int>(fs[f]), ri->status.p, s);
    }
    uint64_t dimsY[2] = {static_cast<uint64_t>(K2), static_cast<uint64_t>(cnt * nt)};
    const CUtensorMap y_hi = bf16_tensor_map(scr.pl_hi.p, 2, dimsY, strk, boxA, swz);
    const CUtensorMap y_lo = bf16_tensor_map(scr.pl_lo.p, 2, dimsY, strk, boxA, swz);
    MoEpi e{};
    e.rows = cnt * nt;
    e.rper = static_cast<int>(nt);
    e.ncol = static_cast<int>(2 * nt);
    e.cmod = static_cast<int>(nt);
    e.ldo = 2 * nt;
    e.conj_odd = 1;
    e.out = m->B.p + P0 * nt * nt * 2;
    launch_step<1>(bn, swz, y_hi, y_lo, cc_hi, cc_lo, e, static_cast<int>(K2), ri->status.p, s);
  }
}

}  // namespace rr
