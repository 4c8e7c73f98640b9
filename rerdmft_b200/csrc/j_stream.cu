// Coulomb streaming passes (see j_stream.cuh).  One producer warp issues 16 KB TMA bulk copies
// into a 4-stage shared-memory ring; 8 consumer warps read them with 128-bit shared loads.
#include <atomic>
#include "j_stream.cuh"
#include "tma_util.cuh"

namespace rr {
namespace {

constexpr int CW = 2048;  // doubles per stage (16 KB)
constexpr int NST = 4;    // ring depth
constexpr int CWARPS = 8;
constexpr int CT = 32 * CWARPS;
constexpr int THREADS = CT + 32;
constexpr int SMEM = NST * CW * 8 + 2 * NST * 8 + CWARPS * 8;
constexpr int ERR_P1_PROD = 1 << 0, ERR_P1_CONS = 1 << 1, ERR_P2_PROD = 1 << 2, ERR_P2_CONS = 1 << 3;

struct P1 {
  JTensor t[2];
  int ntens;
  int64_t naux;
  int nseg[2];
  int64_t seglen[2];
  int segtot;
  int64_t items;
  double* gpart;
  int* err;
  const int* skip;
};

struct P2 {
  JTensor t[2];
  int ntens;
  int64_t naux;
  int segtot;
  int64_t ncol[2];
  int nrange;
  int64_t rp;  // aux rows per range
  int64_t items;
  int64_t jstride;  // len0 + len1
  const double* gpart;
  double* jpart;
  int* err;
  const double* alt;
  int alt_seg;
  const int* alt_flag;
};

__device__ __forceinline__ int64_t min64(int64_t a, int64_t b) { return a < b ? a : b; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void decode1(const P1& p, int64_t it, int& tau, int64_t& P, int& s, int64_t& kb,
                                        int64_t& ke) {
  P = it / p.segtot;
  s = static_cast<int>(it % p.segtot);
  tau = s < p.nseg[0] ? 0 : 1;
  const int seg = tau ? s - p.nseg[0] : s;
  kb = seg * p.seglen[tau];
  ke = min64(p.t[tau].len, kb + p.seglen[tau]);
}

__global__ void __launch_bounds__(THREADS) j_pass1_kernel(const P1 p) {
  if (p.skip && *p.skip) return;
  extern __shared__ __align__(128) unsigned char sm[];
  double* ring = reinterpret_cast<double*>(sm);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + NST * CW * 8);
  uint64_t* empty = full + NST;
  double* red = reinterpret_cast<double*>(empty + NST);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], CWARPS); }
    fence_barrier_init();
  }
  __syncthreads();
  bool dead = false;
  if (warp == CWARPS) {
    if (lane == 0) {
      uint32_t q = 0;
      for (int64_t it = blockIdx.x; it < p.items && !dead; it += gridDim.x) {
        int tau, s;
        int64_t P, kb, ke;
        decode1(p, it, tau, P, s, kb, ke);
        const double* row = p.t[tau].B + P * p.t[tau].pitch;
        for (int64_t k0 = kb; k0 < ke; k0 += CW, ++q) {
          const int st = q % NST;
          if (q >= NST && !mbar_wait(&empty[st], ((q / NST) & 1) ^ 1, p.err, ERR_P1_PROD, dead)) break;
          const uint32_t bytes = static_cast<uint32_t>(round_up_dev(min64(CW, ke - k0), 2) * 8);
          mbar_arrive_expect_tx(&full[st], bytes);
          tma_load_1d(ring + st * CW, row + k0, bytes, &full[st]);
        }
      }
    }
    return;
  }
  const int ct = threadIdx.x;
  uint32_t q = 0;
  for (int64_t it = blockIdx.x; it < p.items; it += gridDim.x) {
    int tau, s;
    int64_t P, kb, ke;
    decode1(p, it, tau, P, s, kb, ke);
    const double* D = p.t[tau].D;
    double acc = 0.0;
    for (int64_t k0 = kb; k0 < ke; k0 += CW, ++q) {
      const int st = q % NST;
      const bool ok = mbar_wait(&full[st], (q / NST) & 1, p.err, ERR_P1_CONS, dead);
      const int64_t len = min64(CW, ke - k0);
      const double2* sb = reinterpret_cast<const double2*>(ring + st * CW);
      const double2* dd = reinterpret_cast<const double2*>(D + k0);
      if (ok) {
#pragma unroll
        for (int v = 0; v < CW / 2 / CT; ++v) {
          const int i2 = ct + v * CT;
          if (2 * i2 < len) {
            const double2 b = sb[i2];
            const double2 d = __ldg(dd + i2);
            acc = fma(b.x, d.x, acc);
            acc = fma(b.y, d.y, acc);
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[st]);
    }
    acc = warp_sum(acc);
    if (lane == 0) red[warp] = acc;
    named_barrier_sync(1, CT);
    if (ct == 0) {
      double t = 0.0;
      for (int w = 0; w < CWARPS; ++w) t += red[w];
      p.gpart[P * p.segtot + s] = t;
    }
    named_barrier_sync(1, CT);
  }
}

__global__ void __launch_bounds__(THREADS) j_pass2_kernel(const P2 p) {
  extern __shared__ __align__(128) unsigned char sm[];
  double* ring = reinterpret_cast<double*>(sm);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + NST * CW * 8);
  uint64_t* empty = full + NST;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], CWARPS); }
    fence_barrier_init();
  }
  __syncthreads();
  const int64_t per_t0 = p.ncol[0] * p.nrange;
  auto decode = [&](int64_t it, int& tau, int64_t& c, int64_t& pb, int64_t& pe) {
    tau = it < per_t0 ? 0 : 1;
    const int64_t j = tau ? it - per_t0 : it;
    const int64_t r = j / p.ncol[tau];
    c = j % p.ncol[tau];
    pb = r * p.rp;
    pe = min64(p.naux, pb + p.rp);
  };
  bool dead = false;
  if (warp == CWARPS) {
    if (lane == 0) {
      uint32_t q = 0;
      for (int64_t it = blockIdx.x; it < p.items && !dead; it += gridDim.x) {
        int tau;
        int64_t c, pb, pe;
        decode(it, tau, c, pb, pe);
        const int64_t k0 = c * CW;
        const uint32_t bytes = static_cast<uint32_t>(round_up_dev(min64(CW, p.t[tau].len - k0), 2) * 8);
        for (int64_t P = pb; P < pe; ++P, ++q) {
          const int st = q % NST;
          if (q >= NST && !mbar_wait(&empty[st], ((q / NST) & 1) ^ 1, p.err, ERR_P2_PROD, dead)) break;
          mbar_arrive_expect_tx(&full[st], bytes);
          tma_load_1d(ring + st * CW, p.t[tau].B + P * p.t[tau].pitch + k0, bytes, &full[st]);
        }
      }
    }
    return;
  }
  const int ct = threadIdx.x;
  const bool use_alt = p.alt_flag && *p.alt_flag;
  const double* gsrc = use_alt ? p.alt : p.gpart;
  const int gseg = use_alt ? p.alt_seg : p.segtot;
  uint32_t q = 0;
  for (int64_t it = blockIdx.x; it < p.items; it += gridDim.x) {
    int tau;
    int64_t c, pb, pe;
    decode(it, tau, c, pb, pe);
    const int64_t k0 = c * CW;
    const int64_t len = min64(CW, p.t[tau].len - k0);
    double2 acc[CW / 2 / CT];
#pragma unroll
    for (int v = 0; v < CW / 2 / CT; ++v) acc[v] = make_double2(0.0, 0.0);
    for (int64_t P = pb; P < pe; ++P, ++q) {
      const int st = q % NST;
      const bool ok = mbar_wait(&full[st], (q / NST) & 1, p.err, ERR_P2_CONS, dead);
      double gam = 0.0;
      const double* gp = gsrc + P * gseg;
      for (int s = 0; s < gseg; ++s) gam += __ldg(gp + s);
      const double2* sb = reinterpret_cast<const double2*>(ring + st * CW);
      if (ok) {
#pragma unroll
        for (int v = 0; v < CW / 2 / CT; ++v) {
          const double2 b = sb[ct + v * CT];
          acc[v].x = fma(gam, b.x, acc[v].x);
          acc[v].y = fma(gam, b.y, acc[v].y);
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[st]);
    }
    const int64_t r = pb / p.rp;
    double* out = p.jpart + r * p.jstride + (tau ? p.t[0].len : 0) + k0;
#pragma unroll
    for (int v = 0; v < CW / 2 / CT; ++v) {
      const int i2 = ct + v * CT;
      if (2 * i2 < len) out[2 * i2] = acc[v].x;
      if (2 * i2 + 1 < len) out[2 * i2 + 1] = acc[v].y;
    }
  }
}

__global__ void j_finish_kernel(JTensor t0, JTensor t1, int ntens, int nrange, int64_t jstride, const double* jpart,
                                double scale) {
  const int64_t total = t0.len + (ntens > 1 ? t1.len : 0);
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < total;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = 0.0;
    for (int r = 0; r < nrange; ++r) s += jpart[r * jstride + k];
    if (k < t0.len) t0.J[k] = scale * s;
    else t1.J[k - t0.len] = scale * s;
  }
}

__global__ void j_gamma_kernel(const double* gpart, int64_t naux, int segtot, double* gamma) {
  for (int64_t P = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; P < naux;
       P += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double g = 0.0;
    for (int s = 0; s < segtot; ++s) g += gpart[P * segtot + s];
    gamma[P] = g;
  }
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

int grid_size(int64_t items, int ctas_per_sm) {
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(items, static_cast<int64_t>(ctas_per_sm) * sm_count())));
}

void set_smem_attr() {
  static std::atomic<bool> done{false};  // host threads may race here: the attribute is idempotent
  if (!done) {
    RR_CUDA(cudaFuncSetAttribute(j_pass1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
    RR_CUDA(cudaFuncSetAttribute(j_pass2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
    done = true;
  }
}

}  // namespace

JPlan j_plan(int ntens, const JTensor* t, int64_t naux, int ctas_per_sm) {
  RR_REQUIRE(ntens >= 1 && ntens <= 2, RR_ERR_ARG, "j_plan: 1 or 2 tensors");
  JPlan pl;
  pl.ntens = ntens;
  pl.naux = naux;
  pl.ctas_per_sm = std::max(1, ctas_per_sm);
  for (int i = 0; i < ntens; ++i) {
    pl.t[i] = t[i];
    RR_REQUIRE(t[i].pitch % 32 == 0 && t[i].pitch >= round_up(t[i].len, 2), RR_ERR_ARG, "j_plan: bad pitch");
    RR_REQUIRE(reinterpret_cast<uintptr_t>(t[i].B) % 256 == 0 && reinterpret_cast<uintptr_t>(t[i].D) % 16 == 0,
               RR_ERR_ARG, "j_plan: misaligned tensor or density");
  }
  const int64_t grid = static_cast<int64_t>(pl.ctas_per_sm) * sm_count();
  // Pass 1: about 16 items per CTA, whole 16 KB chunks per segment.
  for (int i = 0; i < ntens; ++i) {
    const int64_t chunks = std::max<int64_t>(1, (t[i].len + CW - 1) / CW);
    int64_t seg = std::max<int64_t>(1, std::min<int64_t>(chunks, (16 * grid + naux - 1) / std::max<int64_t>(naux, 1)));
    pl.nseg[i] = static_cast<int>(std::min<int64_t>(seg, 64));
  }
  const int64_t ncol = (t[0].len + CW - 1) / CW + (ntens > 1 ? (t[1].len + CW - 1) / CW : 0);
  pl.nrange = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(naux, (4 * grid + ncol - 1) / std::max<int64_t>(ncol, 1))));
  pl.gpart_doubles = naux * (pl.nseg[0] + pl.nseg[1]);
  pl.jpart_doubles = static_cast<int64_t>(pl.nrange) * (t[0].len + (ntens > 1 ? t[1].len : 0));
  return pl;
}

void j_pass1(const JPlan& pl, double* gpart, int* err, cudaStream_t s, const int* skip) {
  if (pl.naux == 0) return;
  set_smem_attr();
  P1 p{};
  p.ntens = pl.ntens;
  p.naux = pl.naux;
  for (int i = 0; i < 2; ++i) {
    p.t[i] = pl.t[i];
    p.nseg[i] = i < pl.ntens ? pl.nseg[i] : 0;
    const int64_t chunks = std::max<int64_t>(1, (pl.t[i].len + CW - 1) / CW);
    p.seglen[i] = p.nseg[i] ? ((chunks + p.nseg[i] - 1) / p.nseg[i]) * CW : CW;
  }
  p.segtot = p.nseg[0] + p.nseg[1];
  p.items = pl.naux * p.segtot;
  p.gpart = gpart;
  p.err = err;
  p.skip = skip;
  j_pass1_kernel<<<grid_size(p.items, pl.ctas_per_sm), THREADS, SMEM, s>>>(p);
  RR_LAUNCH_CHECK();
}

void j_pass2(const JPlan& pl, const double* gpart, double* jpart, int* err, cudaStream_t s, const double* alt,
             int alt_seg, const int* alt_flag) {
  if (pl.naux == 0) return;
  set_smem_attr();
  P2 p{};
  p.ntens = pl.ntens;
  p.naux = pl.naux;
  p.segtot = pl.nseg[0] + pl.nseg[1];
  for (int i = 0; i < 2; ++i) {
    p.t[i] = pl.t[i];
    p.ncol[i] = i < pl.ntens ? (pl.t[i].len + CW - 1) / CW : 0;
  }
  p.nrange = pl.nrange;
  p.rp = (pl.naux + pl.nrange - 1) / pl.nrange;
  p.items = (p.ncol[0] + p.ncol[1]) * pl.nrange;
  p.jstride = pl.t[0].len + (pl.ntens > 1 ? pl.t[1].len : 0);
  p.gpart = gpart;
  p.jpart = jpart;
  p.err = err;
  p.alt = alt;
  p.alt_seg = alt_seg;
  p.alt_flag = alt_flag;
  j_pass2_kernel<<<grid_size(p.items, pl.ctas_per_sm), THREADS, SMEM, s>>>(p);
  RR_LAUNCH_CHECK();
}

void j_finish(const JPlan& pl, const double* jpart, double scale, cudaStream_t s) {
  const int64_t total = pl.t[0].len + (pl.ntens > 1 ? pl.t[1].len : 0);
  if (total == 0) return;
  const int64_t jstride = total;
  // nrange actually used by pass 2 (ranges past naux produce no rows and are never read).
  const int64_t rp = (pl.naux + pl.nrange - 1) / std::max(pl.nrange, 1);
  const int used = pl.naux ? static_cast<int>((pl.naux + rp - 1) / rp) : 0;
  const int blocks = static_cast<int>(std::min<int64_t>(4LL * sm_count(), (total + 255) / 256));
  if (used == 0) {
    RR_CUDA(cudaMemsetAsync(pl.t[0].J, 0, sizeof(double) * pl.t[0].len, s));
    if (pl.ntens > 1) RR_CUDA(cudaMemsetAsync(pl.t[1].J, 0, sizeof(double) * pl.t[1].len, s));
    return;
  }
  j_finish_kernel<<<blocks, 256, 0, s>>>(pl.t[0], pl.t[1], pl.ntens, used, jstride, jpart, scale);
  RR_LAUNCH_CHECK();
}

void j_gamma(const JPlan& pl, const double* gpart, double* gamma, cudaStream_t s) {
  if (pl.naux == 0) return;
  j_gamma_kernel<<<ceil_div(pl.naux, 256), 256, 0, s>>>(gpart, pl.naux, pl.nseg[0] + pl.nseg[1], gamma);
  RR_LAUNCH_CHECK();
}

}  // namespace rr
