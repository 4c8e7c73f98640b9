// Coulomb streaming passes (see j_stream.cuh).  One producer warp issues 16 KB TMA bulk copies
// into a 4-stage shared-memory ring; 8 consumer warps read them with 128-bit shared loads.
#include <atomic>
#include <cfloat>
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
// The pass kernels are held to 48 registers (a few bytes of spills outside the ring loops): one CTA
// then fits on an SM beside two CTAs of the exchange SYRK.
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

__global__ void __maxnreg__(48) j_pass1_kernel(const P1 p) {
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

__global__ void __maxnreg__(48) j_pass2_kernel(const P2 p) {
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

__host__ __device__ inline int64_t out_len(const JTensor& t) { return t.tri_n ? t.tri_n * t.tri_n : t.len; }

// J[t][k] from the pass-2 partials of entry k (packed rows: of entry tri_index(min, max), so both
// triangles get the same sum, added in the same order).
__global__ void j_finish_kernel(JTensor t0, JTensor t1, int ntens, int nrange, int64_t jstride, const double* jpart,
                                double scale) {
  const int64_t out0 = out_len(t0);
  const int64_t total = out0 + (ntens > 1 ? out_len(t1) : 0);
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < total;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const bool second = k >= out0;
    const JTensor& t = second ? t1 : t0;
    const int64_t kk = second ? k - out0 : k;
    int64_t src = second ? t0.len : 0;
    if (t.tri_n) {
      const int64_t q = kk / t.tri_n, a = kk - q * t.tri_n;
      src += q <= a ? tri_index(q, a, t.tri_n) : tri_index(a, q, t.tri_n);
    } else {
      src += kk;
    }
    double s = 0.0;
    for (int r = 0; r < nrange; ++r) s += jpart[r * jstride + src];
    t.J[kk] = scale * s;
  }
}

// Packs the upper triangle of each B^P through 32 x 32 tile pairs (ti <= tj) in shared memory, so
// both the tile and its mirror are read with coalesced loads; *asym = 1 when an element and its
// mirror differ by more than 8 eps of the larger.
__global__ void __launch_bounds__(256) j_pack_kernel(const double* __restrict__ B, int64_t pitch, int64_t naux,
                                                     int64_t n, double* __restrict__ out, int64_t pitch_out,
                                                     int* asym) {
  __shared__ double tu[32][33], tl[32][33];
  const int ntile = static_cast<int>((n + 31) / 32);
  const int ti = static_cast<int>(blockIdx.x) / ntile, tj = static_cast<int>(blockIdx.x) % ntile;
  if (ti > tj) return;
  const int c = threadIdx.x & 31, r0 = threadIdx.x >> 5;
  bool bad = false;
  for (int64_t P = blockIdx.y; P < naux; P += gridDim.y) {
    const double* b = B + P * pitch;
    for (int r = r0; r < 32; r += 8) {
      const int64_t q = ti * 32 + r, a = tj * 32 + c;  // upper tile (q, a)
      tu[r][c] = q < n && a < n ? b[q * n + a] : 0.0;
      const int64_t q2 = tj * 32 + r, a2 = ti * 32 + c;  // mirror tile (a, q), stored transposed
      tl[c][r] = q2 < n && a2 < n ? b[q2 * n + a2] : 0.0;
    }
    __syncthreads();
    double* o = out + P * pitch_out;
    for (int r = r0; r < 32; r += 8) {
      const int64_t q = ti * 32 + r, a = tj * 32 + c;
      if (q < n && a < n && a >= q) {
        const double x = tu[r][c], y = tl[r][c];
        if (!(fabs(x - y) <= 8.0 * DBL_EPSILON * fmax(fabs(x), fabs(y)))) bad = true;
        o[tri_index(q, a, n)] = x;
      }
    }
    __syncthreads();
  }
  if (bad) atomicOr(asym, 1);
}

__global__ void j_fold_kernel(const double* __restrict__ D, int64_t n, double* __restrict__ Dpk) {
  const int64_t n2 = n * n;
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n2;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t q = k / n, a = k - q * n;
    if (a < q) continue;
    Dpk[tri_index(q, a, n)] = a == q ? D[k] : D[k] + D[a * n + q];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && (tri_len(n) & 1)) Dpk[tri_len(n)] = 0.0;
}

__global__ void j_gamma_kernel(const double* gpart, int64_t naux, int segtot, double* gamma) {
  for (int64_t P = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; P < naux;
       P += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double g = 0.0;
    for (int s = 0; s < segtot; ++s) g += gpart[P * segtot + s];
    gamma[P] = g;
  }
}

int sm_count() { return sm_count_current(); }

int grid_size(int64_t items, int ctas_per_sm) {
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(items, static_cast<int64_t>(ctas_per_sm) * sm_count())));
}

void set_smem_attr() {
  static std::atomic<bool> done[kMaxDevices];
  once_per_device(done, [] {
    RR_CUDA(cudaFuncSetAttribute(j_pass1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
    RR_CUDA(cudaFuncSetAttribute(j_pass2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
    // same carveout as the GEMMs they run beside, so an SM can hold both
    RR_CUDA(cudaFuncSetAttribute(j_pass1_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
    RR_CUDA(cudaFuncSetAttribute(j_pass2_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
  });
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
  const int64_t jstride = pl.t[0].len + (pl.ntens > 1 ? pl.t[1].len : 0);
  const int64_t total = out_len(pl.t[0]) + (pl.ntens > 1 ? out_len(pl.t[1]) : 0);
  if (total == 0) return;
  // nrange actually used by pass 2 (ranges past naux produce no rows and are never read).
  const int64_t rp = (pl.naux + pl.nrange - 1) / std::max(pl.nrange, 1);
  const int used = pl.naux ? static_cast<int>((pl.naux + rp - 1) / rp) : 0;
  const int blocks = static_cast<int>(std::min<int64_t>(4LL * sm_count(), (total + 255) / 256));
  if (used == 0) {
    RR_CUDA(cudaMemsetAsync(pl.t[0].J, 0, sizeof(double) * out_len(pl.t[0]), s));
    if (pl.ntens > 1) RR_CUDA(cudaMemsetAsync(pl.t[1].J, 0, sizeof(double) * out_len(pl.t[1]), s));
    return;
  }
  j_finish_kernel<<<blocks, 256, 0, s>>>(pl.t[0], pl.t[1], pl.ntens, used, jstride, jpart, scale);
  RR_LAUNCH_CHECK();
}

bool j_pack_upper(const double* B, int64_t pitch, int64_t naux, int64_t n, DevBuf<double>& out, int64_t& pitch_out,
                  cudaStream_t s) {
  RR_REQUIRE(n >= 1 && naux >= 1 && pitch >= n * n, RR_ERR_ARG, "j_pack_upper: bad shape");
  pitch_out = round_up(tri_len(n), 32);
  out.alloc(static_cast<size_t>(naux * pitch_out));
  RR_CUDA(cudaMemsetAsync(out.p, 0, sizeof(double) * out.n, s));
  DevBuf<int> asym(1);
  RR_CUDA(cudaMemsetAsync(asym.p, 0, sizeof(int), s));
  const int64_t ntile = (n + 31) / 32;
  const dim3 grid(static_cast<unsigned>(ntile * ntile), static_cast<unsigned>(std::min<int64_t>(naux, 65535)));
  j_pack_kernel<<<grid, 256, 0, s>>>(B, pitch, naux, n, out.p, pitch_out, asym.p);
  RR_LAUNCH_CHECK();
  int h = 0;
  RR_CUDA(cudaMemcpyAsync(&h, asym.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  RR_CUDA(cudaStreamSynchronize(s));
  if (h) {
    out.release();
    pitch_out = 0;
    return false;
  }
  return true;
}

void j_fold_density(const double* D, int64_t n, double* Dpk, cudaStream_t s) {
  const int blocks = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(2LL * sm_count(), (n * n + 255) / 256)));
  j_fold_kernel<<<blocks, 256, 0, s>>>(D, n, Dpk);
  RR_LAUNCH_CHECK();
}

void j_gamma(const JPlan& pl, const double* gpart, double* gamma, cudaStream_t s) {
  if (pl.naux == 0) return;
  j_gamma_kernel<<<ceil_div(pl.naux, 256), 256, 0, s>>>(gpart, pl.naux, pl.nseg[0] + pl.nseg[1], gamma);
  RR_LAUNCH_CHECK();
}

}  // namespace rr
