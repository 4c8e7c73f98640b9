// FP64 DMMA GEMM: multistage cp.async pipeline (3 stages of 16-deep k tiles), warp tiles of
// (MT*8) x (NT*8) built from mma.sync.m8n8k4.f64, optional complex (4M) accumulation, split-K
// with a fixed-order reduction (bit-identical results run to run), and upper-triangle-only
// scheduling for symmetric / Hermitian outputs.
#include <atomic>
#include <cstdlib>

#include "gemm_tile.cuh"

namespace rr {
namespace {

using namespace gk;

template <int MT, int NT, int WM, int WN, bool AK, bool BKM, bool CPLX, int V, bool EDOT = false>
__global__ void __launch_bounds__(32 * WM * WN) dgemm_kernel(const Params p) {
  using CF = Cfg<MT, NT, WM, WN, AK, BKM, CPLX>;
  extern __shared__ __align__(16) double smem[];
  const int64_t n0 = static_cast<int64_t>(blockIdx.x) * CF::BN;
  const int64_t m0 = static_cast<int64_t>(blockIdx.y) * CF::BM;
  if (p.upper_only && m0 > n0 + CF::BN - 1) return;
  const int64_t bz = blockIdx.z;
  const int64_t b = bz / p.splits;
  dgemm_tile<MT, NT, WM, WN, AK, BKM, CPLX, V, EDOT>(p, n0, m0, bz, smem,
                                                      b * (gridDim.x * gridDim.y) + blockIdx.y * gridDim.x + blockIdx.x);
}

template <int PL>
__global__ void splitk_reduce_kernel(const Params p) {
  const int64_t total = p.batch * p.M * p.N;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x)
    splitk_reduce_elem<PL>(p, idx);
}

template <int PL>
__global__ void mirror_kernel(double* C, int64_t n, int64_t ldc, int64_t strideC, int64_t batch, int mode) {
  const int64_t total = batch * n * n;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x)
    mirror_elem<PL>(C, n, ldc, strideC, mode, idx);
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
