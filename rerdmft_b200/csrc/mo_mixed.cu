// Split-BF16 MO three-index transform on the 5th-generation tensor cores (RR_PREC_MIXED of
// rr_mo_build_nonrel): B_mo^P = C^T B^P C for every aux index P.
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
// drain TMEM (lanes 32 w .. 32 w + 31), warp 4 lane 0 issues the TMA ring, warp 5 lane 0 the MMAs.
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

// Output of one step.  Row R of the flat product is (P, r) with P = R / n, r = R % n; column c < n.
//   EPI 0: hi/lo[(P n + c) ldq + r] = split(value)      (Yt[P][c][r])
//   EPI 1: out[R n + c] = value                          (B_mo[P][r][c])
struct MoEpi {
  int64_t rows;  // naux * n
  int n;
  int64_t ldq;
  __nv_bfloat16* hi;
  __nv_bfloat16* lo;
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
                   const MoEpi e, int nkb, int64_t rtiles, int ntn, int* err) {
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
      constexpr uint32_t idesc = idesc_bf16_f32(BM, BN);
      uint32_t q = 0, j = 0;
      for (int64_t item = blockIdx.x; item < total; item += gridDim.x, ++j) {
        const uint32_t b = j & 1;
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
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
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
        const int64_t P = live ? R / e.n : 0;
        const int r = live ? static_cast<int>(R - P * e.n) : 0;
        // Fast paths write through the staging tile: EPI 0 as 16-byte runs of 8 consecutive r of one P (all 32
        // rows live and in one P, r 8-aligned), EPI 1 as whole 128- / 256-byte row segments (n even).
        const int64_t P0 = R0 / e.n;
        const int a0 = static_cast<int>(R0 - P0 * e.n);
        const bool rows_ok = R0 + 31 < e.rows;
        const bool fast0 = rows_ok && a0 + 31 < e.n && (a0 & 7) == 0 && (e.n & 7) == 0;
        const bool fast1 = rows_ok && (e.n & 1) == 0;
        for (int c0 = 0; c0 < BN && n0 + c0 < e.n; c0 += 32) {  // warp-uniform bounds
          const int W = c0 + 32 <= BN ? 32 : 16;                  // BN is a multiple of 16
          float v[32];
          if (W == 32) tmem_ld32(tmem + lane_base + b * CF::BNP + c0, v);
          else tmem_ld16(tmem + lane_base + b * CF::BNP + c0, v);
          const int cb = n0 + c0;
          const int cw = min(W, e.n - cb);  // valid columns of this chunk
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
                const int64_t o = (P0 * e.n + cb + jc) * e.ldq + a0 + 8 * g;
                *reinterpret_cast<uint4*>(e.hi + o) = make_uint4(h[0], h[1], h[2], h[3]);
                *reinterpret_cast<uint4*>(e.lo + o) = make_uint4(l[0], l[1], l[2], l[3]);
              }
            } else if (live) {
#pragma unroll
              for (int t = 0; t < 32; ++t) {
                if (t >= cw) continue;
                const int64_t o = (P * e.n + cb + t) * e.ldq + r;
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
                                                 static_cast<double>(sw[rr * 33 + 2 * cp + 1]));
                  *reinterpret_cast<double2*>(e.out + (R0 + rr) * e.n + cb + 2 * cp) = d;
                }
              } else {
#pragma unroll
                for (int t = 0; t < 32; t += 2)
                  if (t < cw)
                    *reinterpret_cast<double2*>(e.out + R * e.n + cb + t) =
                        make_double2(static_cast<double>(v[t]), static_cast<double>(v[t + 1]));
              }
            } else if (live) {
#pragma unroll
              for (int t = 0; t < 32; ++t)
                if (t < cw) e.out[R * e.n + cb + t] = static_cast<double>(v[t]);
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
               const MoEpi& e, int nkb, int* err, cudaStream_t s) {
  using CF = MoCfg<BN, STAGES, SWZ>;
  auto kern = umma_mo_kernel<BN, STAGES, EPI, SWZ>;
  static std::atomic<bool> attr[kMaxDevices];
  once_per_device(attr, [&] { RR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, CF::SMEM)); });
  const int64_t rtiles = (e.rows + BM - 1) / BM;
  const int ntn = (e.n + BN - 1) / BN;
  const int64_t items = rtiles * ntn;
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(items, sm_count_current())));
  kern<<<grid, MO_THREADS, CF::SMEM, s>>>(a_hi, a_lo, b_hi, b_lo, e, nkb, rtiles, ntn, err);
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
                 const CUtensorMap& b_lo, const MoEpi& e, int nkb, int* err, cudaStream_t s) {
  if (swz == 128) {
    switch (bn) {
      case 128: return launch_mo<128, 3, EPI, 128>(a_hi, a_lo, b_hi, b_lo, e, nkb, err, s);
      case 144: return launch_mo<144, 3, EPI, 128>(a_hi, a_lo, b_hi, b_lo, e, nkb, err, s);
      default: return launch_mo<208, 2, EPI, 128>(a_hi, a_lo, b_hi, b_lo, e, nkb, err, s);
    }
  }
  switch (bn) {
    case 32: return launch_mo<32, 8, EPI, 64>(a_hi, a_lo, b_hi, b_lo, e, nkb, err, s);
    case 64: return launch_mo<64, 8, EPI, 64>(a_hi, a_lo, b_hi, b_lo, e, nkb, err, s);
    case 112: return launch_mo<112, 6, EPI, 64>(a_hi, a_lo, b_hi, b_lo, e, nkb, err, s);
    case 128: return launch_mo<128, 6, EPI, 64>(a_hi, a_lo, b_hi, b_lo, e, nkb, err, s);
    case 144: return launch_mo<144, 6, EPI, 64>(a_hi, a_lo, b_hi, b_lo, e, nkb, err, s);
    case 208: return launch_mo<208, 4, EPI, 64>(a_hi, a_lo, b_hi, b_lo, e, nkb, err, s);
    default: return launch_mo<256, 4, EPI, 64>(a_hi, a_lo, b_hi, b_lo, e, nkb, err, s);
  }
}

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

  int bn = pick_bn(n);
  if (const char* v = std::getenv("RR_MO_BN")) {  // measurement: force a column tile width
    const int f = std::atoi(v);
    RR_REQUIRE(f == 32 || f == 64 || f == 112 || f == 128 || f == 144 || f == 208 || f == 256, RR_ERR_ARG,
               "RR_MO_BN: one of 32, 64, 112, 128, 144, 208, 256");
    bn = f;
  }
  // 128-byte swizzle (64-deep K blocks) where it is instantiated; the 64-byte swizzle's deeper ring measured
  // slower at n = 400 (1.371 against 1.321 ms per build with BN = 208).
  int swz = (bn == 128 || bn == 144 || bn == 208) ? 128 : 64;
  if (const char* v = std::getenv("RR_MO_SWZ")) {  // measurement: force the swizzle
    swz = std::atoi(v);
    RR_REQUIRE((swz == 64) || (swz == 128 && (bn == 128 || bn == 144 || bn == 208)), RR_ERR_ARG,
               "RR_MO_SWZ: 64, or 128 with a column tile of 128, 144 or 208");
  }
  const int BK = swz / 2;
  const int nkb = static_cast<int>((n + BK - 1) / BK);
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
  e.n = static_cast<int>(n);
  e.ldq = ldq;
  e.hi = reinterpret_cast<__nv_bfloat16*>(scr.pl_hi.p);
  e.lo = reinterpret_cast<__nv_bfloat16*>(scr.pl_lo.p);
  e.out = m->B.p;
  launch_step<0>(bn, swz, bt_hi, bt_lo, c_hi, c_lo, e, nkb, ri->status.p, s);  // Yt = (B^P^T C)^T, split
  launch_step<1>(bn, swz, y_hi, y_lo, c_hi, c_lo, e, nkb, ri->status.p, s);    // B_mo^P = C^T B^P C, FP64
}

}  // namespace rr
