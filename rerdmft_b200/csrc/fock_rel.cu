// Relativistic RI Fock builds: X2C (2 spin blocks) and the 4-component UKB/RKB build (4 blocks).
//
// References: src/X2C_DHF/X2C_FockMatrixRi.cpp:79-205 (x2cFockMatrix),
// src/UKB/UkbFockMatrixRi.cpp:35-183 (riFockTwoElectronDirect), :185-216 (rkbFockMatrix).
//
// The 3-center tensors are real and the coefficients complex.  As in the reference, the complex
// half-transform is carried out as real GEMMs on split real/imaginary rows; the exchange blocks
// K_fu = V_f^dagger V_u (V_f = tmp_f over all P, flattened to (naux*r) x fs_f) then map onto
// real FP64 DMMA GEMMs:  Re K = [Re V_f; Im V_f]^T [Re V_u; Im V_u]  (one GEMM: the two planes are
// stored back to back) and  Im K = Re V_f^T Im V_u - Im V_f^T Re V_u  (two GEMMs).  Diagonal
// blocks f = u compute only upper tiles (Re symmetric, Im antisymmetric) and mirror.
#include <algorithm>
#include <array>

#include "ri_store.cuh"

namespace rr {

void projector_ct(rr_ri_store* h, const double* A, const double* Pe, const double* X, int64_t n, int64_t n_eff,
                  int64_t r, bool cplx, double* Ct, cudaStream_t s);
void prof_mark(rr_ri_store* h, int i, cudaStream_t s);

namespace {

int blocks_for(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 1184))); }

// Real part of the spin-summed density of two same-size flavour blocks into a pitched buffer:
// out[a*fs + b] = Re(P(o0+a, o0+b) + P(o1+a, o1+b)), P complex n x n.
__global__ void spin_sum_kernel(double* out, const double* P, int64_t n, int64_t o0, int64_t o1, int64_t fs) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < fs * fs;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t a = idx / fs, b = idx % fs;
    out[idx] = P[((o0 + a) * n + o0 + b) * 2] + P[((o1 + a) * n + o1 + b) * 2];
  }
}

// Planar split of one flavour's columns of Ct (r x ntot complex): out (2r x fs) real,
// rows [0, r) real parts, rows [r, 2r) imaginary parts.
__global__ void split_rows_kernel(double* out, const double* Ct, int64_t r, int64_t ntot, int64_t off, int64_t fs) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < 2 * r * fs;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx / fs, a = idx % fs;
    const int64_t ii = i < r ? i : i - r;
    out[idx] = Ct[(ii * ntot + off + a) * 2 + (i < r ? 0 : 1)];
  }
}

// G (complex ntot x ntot) block (f,u): G(of+a, ou+b) = sgn (Kre + i Kim)(a,b), and for f != u also
// G(ou+b, of+a) = sgn conj(K(a,b)).  diag_j (real fs x fs) is added on a diagonal block.
__global__ void place_block_kernel(double* G, int64_t ntot, int64_t of, int64_t ou, int64_t fsf, int64_t fsu,
                                   const double* Kre, const double* Kim, const double* diag_j, int both, double sgn) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < fsf * fsu;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t a = idx / fsu, b = idx % fsu;
    const double re = sgn * Kre[idx], im = sgn * Kim[idx];
    double* g = G + ((of + a) * ntot + ou + b) * 2;
    g[0] = re + (diag_j ? diag_j[idx] : 0.0);
    g[1] = im;
    if (both) {
      double* gt = G + ((ou + b) * ntot + of + a) * 2;
      gt[0] = re;
      gt[1] = -im;
    }
  }
}

// Gauss (3M) planes of one flavour's half-transform T = [Re (kk x fs) | Im (kk x fs)]:
// minus = Re - Im and plus = Re + Im (either may be null).
__global__ void plane_pm_kernel(const double* T, int64_t cnt, double* minus, double* plus) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < cnt;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double re = T[i], im = T[cnt + i];
    if (minus) minus[i] = re - im;
    if (plus) plus[i] = re + im;
  }
}

// 3M combine: Re K = P1 + P2, Im K = P3 - P1 + P2 with P1 in Kre, P2 in K2, P3 in Kim.
__global__ void combine_3m_kernel(double* Kre, double* Kim, const double* K2, int64_t count) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double p1 = Kre[i], p2 = K2[i];
    Kim[i] = Kim[i] - p1 + p2;
    Kre[i] = p1 + p2;
  }
}

// G = -K (count doubles).
__global__ void neg_copy_kernel(double* G, const double* K, int64_t count) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    G[i] = -K[i];
}

// Real part of the diagonal block (off, off) of G (complex ntot x ntot) += J (real fs x fs).
__global__ void add_j_block_kernel(double* G, int64_t ntot, int64_t off, int64_t fs, const double* J) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < fs * fs;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t a = idx / fs, b = idx % fs;
    G[((off + a) * ntot + off + b) * 2] += J[idx];
  }
}

// Ct (r x ntot complex) = diag(sqrt(occ)) C^dagger for C (ntot x r complex).
__global__ void ct_from_occupied_kernel(double* Ct, const double* C, const double* occ, int64_t ntot, int64_t r) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < r * ntot;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx / ntot, a = idx % ntot;
    const double w = sqrt(occ[i]);
    Ct[idx * 2] = w * C[(a * r + i) * 2];
    Ct[idx * 2 + 1] = -w * C[(a * r + i) * 2 + 1];
  }
}

// out = h + G  (complex, interleaved; count complex entries)
__global__ void add_kernel(double* out, const double* h, const double* G, int64_t count2) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count2;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = h[i] + G[i];
}

// Deterministic two-stage sums for the energy-only evaluation: EN_CTAS CTAs write one partial each
// over fixed chunks, one CTA adds them in order.
constexpr int EN_CTAS = 256;

__device__ __forceinline__ double en_block_sum(double v) {
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += red[w];
  __syncthreads();
  return t;
}

// part[b] = this CTA's share of sum_P sum_ij (Q11 + Q22)_ij^2 + (Q21 - Q12)_ij^2, Q^P = [Qtop; Qbot]
// (2r x 2r per aux row: Qtop = [Re T Cr^T | Re T Ci^T], Qbot = [Im T Cr^T | Im T Ci^T]), i.e.
// ||M^P||_F^2 with M^P = sum_f c_f B^P c_f^dagger = (Q11 + Q22) + i (Q21 - Q12).
__global__ void exchange_energy_partial_kernel(const double* Q, int64_t naux, int64_t r, double* part) {
  const int64_t cnt = naux * r * r, per = (cnt + gridDim.x - 1) / gridDim.x;
  const int64_t beg = blockIdx.x * per, end = beg + per < cnt ? beg + per : cnt;
  double acc = 0.0;
  for (int64_t idx = beg + threadIdx.x; idx < end; idx += blockDim.x) {
    const int64_t P = idx / (r * r), e = idx % (r * r), i = e / r, j = e % r;
    const double* q = Q + P * 4 * r * r;
    const double q11 = q[i * 2 * r + j], q12 = q[i * 2 * r + r + j];
    const double q21 = q[(r + i) * 2 * r + j], q22 = q[(r + i) * 2 * r + r + j];
    const double re = q11 + q22, im = q21 - q12;
    acc += re * re + im * im;
  }
  acc = en_block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// part[b] = this CTA's share of sum_k D[k] J[k] over cnt entries (sum of D[k]^2 when J is null).
__global__ void dot_partial_kernel(const double* D, const double* J, int64_t cnt, double* part) {
  const int64_t per = (cnt + gridDim.x - 1) / gridDim.x;
  const int64_t beg = blockIdx.x * per, end = beg + per < cnt ? beg + per : cnt;
  double acc = 0.0;
  for (int64_t idx = beg + threadIdx.x; idx < end; idx += blockDim.x) acc += D[idx] * (J ? J[idx] : D[idx]);
  acc = en_block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// out[0] = scale * sum of the `np` partials (one CTA, fixed order); with accumulate, out[0] += that.
__global__ void sum_partials_kernel(const double* part, int np, double scale, double* out, int accumulate) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) acc += part[i];
  acc = en_block_sum(acc);
  if (threadIdx.x == 0) out[0] = (accumulate ? out[0] : 0.0) + scale * acc;
}

struct Flavours {
  int nf = 0;
  std::array<int64_t, 4> off{}, fs{};
  std::array<int, 4> tens{};
};

}  // namespace

void coulomb_async_multi(rr_ri_store* h, int ntens, const double* const* Dp, double* const* J, cudaStream_t s);

void dot_sum(const double* a, const double* b, int64_t cnt, double scale, double* out, bool accumulate, double* part,
             cudaStream_t s) {
  dot_partial_kernel<<<EN_CTAS, 256, 0, s>>>(a, b, cnt, part);
  RR_LAUNCH_CHECK();
  sum_partials_kernel<<<1, 256, 0, s>>>(part, EN_CTAS, scale, out, accumulate ? 1 : 0);
  RR_LAUNCH_CHECK();
}

// Two-electron matrix G (complex ntot x ntot) = J - K for the given flavours from Ct (r x ntot,
// complex), the reference's c_t of all flavours side by side.  Pdens: pitched real spin-summed
// densities per tensor (J input).  Writes G.  With rb the exchange goes through the handle's
// accumulator (RelBuild).
void two_electron_rel(rr_ri_store* h, const Flavours& fl, int64_t ntot, const double* Ct, int64_t r,
                      const double* const* Dp, double* G, cudaStream_t s, const RelBuild* rb) {
  const int64_t naux = h->naux;
  const int ntens = h->ntens;
  std::array<int64_t, 2> nt = {h->n, h->ns};
  // J (side stream) into per-tensor J buffers
  double *J[2] = {nullptr, nullptr}, *Cs[4], *Kre, *Kim;
  int64_t fsmax = 0;
  for (int f = 0; f < fl.nf; ++f) fsmax = std::max(fsmax, fl.fs[f]);
  Arena ar(&h->mats);
  for (int t = 0; t < ntens; ++t) ar.request(&J[t], nt[t] * nt[t]);
  for (int f = 0; f < fl.nf; ++f) ar.request(&Cs[f], 2 * std::max<int64_t>(r, 1) * fl.fs[f]);
  double* K2;
  ar.request(&Kre, fsmax * fsmax);
  ar.request(&Kim, fsmax * fsmax);
  ar.request(&K2, fsmax * fsmax);
  ar.commit();
  coulomb_async_multi(h, ntens, Dp, J, s);
  const bool energy_only = rb && rb->energy;
  RR_REQUIRE(!energy_only || !rb->mixed, RR_ERR_STATE, "two_electron_rel: the energy-only evaluation is FP64");
  if (rb && !energy_only) {
    h->inc_k.ensure(static_cast<size_t>(2 * ntot * ntot));
    if (rb->mixed) {
      const bool incr = rb->incremental && h->inc_r == r && h->inc_ld == ntot && r > 0;
      ExFlavours ef;
      ef.nf = fl.nf;
      for (int f = 0; f < fl.nf; ++f) {
        ef.off[f] = fl.off[f];
        ef.fs[f] = fl.fs[f];
        ef.tens[f] = fl.tens[f];
      }
      for (int t = 0; t < ntens; ++t) mixed_prepare(h->mixed[t], h->B[t].p, h->pitch[t], nt[t], naux, s);
      prof_mark(h, 2, s);
      mixed_exchange_general(h->mixed, h->mscr, ef, naux, Ct, incr ? h->inc_ct.p : nullptr, ntot, r, true, h->inc_k.p,
                             ntot, incr, h->status.p, s);
      prof_mark(h, 3, s);
    }
  }
  const bool fp64_k = !rb || !rb->mixed;
  double* Gk = rb ? h->inc_k.p : G;  // where the FP64 blocks land
  if (fp64_k && !energy_only) RR_CUDA(cudaMemsetAsync(Gk, 0, sizeof(double) * 2 * ntot * ntot, s));
  // T planes: flavour f occupies [Re (naux*r*fs) | Im (naux*r*fs)]; the off-diagonal blocks (f < u)
  // use Gauss's three products, with Re - Im of every flavour that is an f and Re + Im of every
  // flavour that is a u of such a block.
  std::array<double*, 4> T{}, Tm{}, Tp{};
  int64_t tsize = 0;
  for (int f = 0; f < fl.nf; ++f) tsize += 2 * naux * r * fl.fs[f];
  if (!energy_only)
    for (int f = 0; f < fl.nf; ++f) tsize += (f + 1 < fl.nf ? naux * r * fl.fs[f] : 0) + (f > 0 ? naux * r * fl.fs[f] : 0);
  // energy-only: the 2r x 2r products Q^P of every aux row follow the planes
  const int64_t qsize = energy_only ? round_up(naux * 4 * r * r, 32) : 0;
  if (fp64_k && r > 0 && naux > 0) {
    h->T.ensure(static_cast<size_t>(round_up(tsize, 32) + qsize + EN_CTAS));
    int64_t o = 0;
    for (int f = 0; f < fl.nf; ++f) { T[f] = h->T.p + o; o += 2 * naux * r * fl.fs[f]; }
    for (int f = 0; f < fl.nf; ++f) {
      if (f + 1 < fl.nf) { Tm[f] = h->T.p + o; o += naux * r * fl.fs[f]; }
      if (f > 0) { Tp[f] = h->T.p + o; o += naux * r * fl.fs[f]; }
    }
    for (int f = 0; f < fl.nf; ++f) {
      split_rows_kernel<<<blocks_for(2 * r * fl.fs[f]), 256, 0, s>>>(Cs[f], Ct, r, ntot, fl.off[f], fl.fs[f]);
      RR_LAUNCH_CHECK();
      const int t = fl.tens[f];
      GemmDesc ht;
      ht.M = 2 * r; ht.N = fl.fs[f]; ht.K = fl.fs[f];
      ht.A = Cs[f]; ht.lda = fl.fs[f];
      ht.B = h->B[t].p; ht.ldb = fl.fs[f]; ht.strideB = h->pitch[t];
      ht.C = T[f]; ht.ldc = fl.fs[f]; ht.strideC = r * fl.fs[f];
      ht.c_plane_rows = r; ht.c_plane_stride = naux * r * fl.fs[f];
      ht.batch = naux;
      gemm(ht, s);
    }
    for (int f = 0; f < fl.nf && fl.nf > 1 && !energy_only; ++f) {
      const int64_t cnt = naux * r * fl.fs[f];
      plane_pm_kernel<<<blocks_for(cnt), 256, 0, s>>>(T[f], cnt, Tm[f], Tp[f]);
      RR_LAUNCH_CHECK();
    }
  }
  if (energy_only) {
    // E_K = sum_P ||sum_f (c_f B^P) c_f^dagger||_F^2 from the half-transform planes: per flavour
    // Qtop^P += Re T_f^P Cs_f^T and Qbot^P += Im T_f^P Cs_f^T (Cs_f = [Re c_f; Im c_f]), r x 2r each
    double* part = h->T.p + round_up(tsize, 32) + qsize;
    if (r > 0 && naux > 0) {
      double* Q = h->T.p + round_up(tsize, 32);
      for (int f = 0; f < fl.nf; ++f)
        for (int plane = 0; plane < 2; ++plane) {
          GemmDesc q;
          q.M = r; q.N = 2 * r; q.K = fl.fs[f];
          q.A = T[f] + plane * naux * r * fl.fs[f]; q.lda = fl.fs[f]; q.strideA = r * fl.fs[f];
          q.B = Cs[f]; q.ldb = fl.fs[f]; q.opB = Op::T; q.strideB = 0;
          q.C = Q + plane * r * 2 * r; q.ldc = 2 * r; q.strideC = 4 * r * r;
          q.batch = naux;
          q.beta = f > 0 ? 1.0 : 0.0;
          gemm(q, s);
        }
      exchange_energy_partial_kernel<<<EN_CTAS, 256, 0, s>>>(Q, naux, r, part);
      RR_LAUNCH_CHECK();
      sum_partials_kernel<<<1, 256, 0, s>>>(part, EN_CTAS, 1.0, rb->energy + 1, 0);
      RR_LAUNCH_CHECK();
    } else {
      RR_CUDA(cudaMemsetAsync(rb->energy + 1, 0, sizeof(double), s));
    }
    // E_J = 1/2 sum_t <D_t, J_t> once the J passes are done
    RR_CUDA(cudaStreamWaitEvent(s, h->ctx.join, 0));
    h->work.ensure(static_cast<size_t>(std::max<int64_t>(static_cast<int64_t>(h->work.n), EN_CTAS)));
    double* jpart = h->work.p;
    for (int t = 0; t < ntens; ++t) dot_sum(Dp[t], J[t], nt[t] * nt[t], 0.5, rb->energy, t > 0, jpart, s);
    return;
  }
  if (fp64_k) prof_mark(h, 2, s);
  for (int f = 0; f < fl.nf && fp64_k; ++f)
    for (int u = f; u < fl.nf; ++u) {
      const int64_t ff = fl.fs[f], fu = fl.fs[u];
      if (r > 0 && naux > 0) {
        const int64_t kk = naux * r;
        GemmDesc g;
        g.M = ff; g.N = fu;
        g.opA = Op::T; g.lda = ff; g.ldb = fu; g.ldc = fu;
        if (f == u) {
          // Hermitian diagonal block, upper tiles: Re K = [Re; Im]^T [Re; Im] (symmetric),
          // Im K = Re^T Im - Im^T Re (antisymmetric)
          g.K = 2 * kk; g.A = T[f]; g.B = T[u]; g.C = Kre; g.mirror = 1;
          int64_t want = gemm_work_doubles(g);
          h->work.ensure(static_cast<size_t>(std::max<int64_t>(want, 1)));
          gemm(g, s, h->work.p, static_cast<int64_t>(h->work.n));
          g.K = kk; g.A = T[f]; g.B = T[u] + kk * fu; g.C = Kim; g.alpha = 1.0; g.beta = 0.0;
          g.mirror = -1;
          gemm(g, s, h->work.p, static_cast<int64_t>(h->work.n));
          g.A = T[f] + kk * ff; g.B = T[u]; g.alpha = -1.0; g.beta = 1.0;
          gemm(g, s, h->work.p, static_cast<int64_t>(h->work.n));
        } else {
          // Gauss: P1 = Re_f^T Re_u, P2 = Im_f^T Im_u, P3 = (Re - Im)_f^T (Re + Im)_u;
          // Re K = P1 + P2, Im K = P3 - P1 + P2 (three products instead of four)
          g.K = kk; g.A = T[f]; g.B = T[u]; g.C = Kre;
          int64_t want = gemm_work_doubles(g);
          h->work.ensure(static_cast<size_t>(std::max<int64_t>(want, 1)));
          gemm(g, s, h->work.p, static_cast<int64_t>(h->work.n));
          g.A = T[f] + kk * ff; g.B = T[u] + kk * fu; g.C = K2;
          gemm(g, s, h->work.p, static_cast<int64_t>(h->work.n));
          g.A = Tm[f]; g.B = Tp[u]; g.C = Kim;
          gemm(g, s, h->work.p, static_cast<int64_t>(h->work.n));
          combine_3m_kernel<<<blocks_for(ff * fu), 256, 0, s>>>(Kre, Kim, K2, ff * fu);
          RR_LAUNCH_CHECK();
        }
      } else {
        RR_CUDA(cudaMemsetAsync(Kre, 0, sizeof(double) * ff * fu, s));
        RR_CUDA(cudaMemsetAsync(Kim, 0, sizeof(double) * ff * fu, s));
      }
      const bool add_j = f == u && !rb;
      if (add_j) RR_CUDA(cudaStreamWaitEvent(s, h->ctx.join, 0));  // J needed on the diagonal blocks
      place_block_kernel<<<blocks_for(ff * fu), 256, 0, s>>>(Gk, ntot, fl.off[f], fl.off[u], ff, fu, Kre, Kim,
                                                              add_j ? J[fl.tens[f]] : nullptr, f != u, rb ? 1.0 : -1.0);
      RR_LAUNCH_CHECK();
    }
  if (fp64_k) prof_mark(h, 3, s);
  if (rb) {
    // G = J - K from the accumulator; remember c_t for the next incremental build
    neg_copy_kernel<<<blocks_for(2 * ntot * ntot), 256, 0, s>>>(G, h->inc_k.p, 2 * ntot * ntot);
    RR_LAUNCH_CHECK();
    RR_CUDA(cudaStreamWaitEvent(s, h->ctx.join, 0));
    for (int f = 0; f < fl.nf; ++f) {
      add_j_block_kernel<<<blocks_for(fl.fs[f] * fl.fs[f]), 256, 0, s>>>(G, ntot, fl.off[f], fl.fs[f], J[fl.tens[f]]);
      RR_LAUNCH_CHECK();
    }
    h->inc_ct.ensure(static_cast<size_t>(std::max<int64_t>(2 * r * ntot, 1)));
    if (r > 0) RR_CUDA(cudaMemcpyAsync(h->inc_ct.p, Ct, sizeof(double) * 2 * r * ntot, cudaMemcpyDeviceToDevice, s));
    h->inc_r = r;
    h->inc_ld = ntot;
  }
}

// With `proj` (device, n_eff x n_eff, a rank-proj_rank orthogonal projector in the orthonormal basis
// of X whose X proj X^dagger is P, as the SCF loop has it from SP2) the occupied spinors come from
// that projector directly instead of being recovered from P.
void fock_x2c(rr_ri_store* h, const double* hc, const double* P, const double* S, const double* X, int64_t n_eff,
              double* F, const rr_opts* o, const RelBuild* rb, const double* proj, int64_t proj_rank) {
  RR_REQUIRE(h->ntens == 1, RR_ERR_STATE, "rr_ri_fock_x2c: handle holds a 4-component store");
  const int64_t nl = h->n, n = 2 * nl, nn2 = n * n * 2;
  RR_REQUIRE(n_eff >= 0 && n_eff <= n, RR_ERR_ARG, "rr_ri_fock_x2c: n_eff out of range");
  const bool host = !o || o->mem == RR_MEM_HOST;
  cudaStream_t s = call_stream(h, o);
  const int64_t pitch = round_up(std::max<int64_t>(nl * nl, 2), 32);
  double *Pd = nullptr, *hd = nullptr, *Sd = nullptr, *Xd = nullptr, *Fd = nullptr, *Dp, *Ct, *G;
  // This call's matrices live in `solver_w`: two_electron_rel and occupied_ct re-carve `mats` and
  // `solver_a` for their own intermediates.
  Arena ar(&h->solver_w);
  ar.request(&Dp, pitch);
  ar.request(&Ct, 2 * n * std::max<int64_t>(n_eff, 1));
  ar.request(&G, nn2);
  if (host) {
    ar.request(&hd, nn2);
    ar.request(&Pd, nn2);
    ar.request(&Sd, nn2);
    ar.request(&Xd, 2 * n * n_eff);
    ar.request(&Fd, nn2);
  }
  ar.commit();
  if (!host) {
    hd = const_cast<double*>(hc); Pd = const_cast<double*>(P); Sd = const_cast<double*>(S); Xd = const_cast<double*>(X);
    Fd = F;
  }
  prof_mark(h, 0, s);
  if (host) {
    copy_in(hd, hc, nn2, true, s);
    copy_in(Pd, P, nn2, true, s);
    copy_in(Sd, S, nn2, true, s);
    copy_in(Xd, X, 2 * n * n_eff, true, s);
  }
  RR_CUDA(cudaMemsetAsync(Dp, 0, sizeof(double) * pitch, s));
  spin_sum_kernel<<<blocks_for(nl * nl), 256, 0, s>>>(Dp, Pd, n, 0, nl, nl);
  RR_LAUNCH_CHECK();
  int64_t r = proj_rank;
  if (proj) projector_ct(h, proj, nullptr, Xd, n, n_eff, r, true, Ct, s);
  else r = occupied_ct(h, Xd, Sd, Pd, n, n_eff, 1.0, true, true, Ct, s);
  prof_mark(h, 1, s);
  Flavours fl;
  fl.nf = 2;
  fl.off = {0, nl, 0, 0};
  fl.fs = {nl, nl, 0, 0};
  fl.tens = {0, 0, 0, 0};
  const double* dps[1] = {Dp};
  two_electron_rel(h, fl, n, Ct, r, dps, G, s, rb);
  if (!(rb && rb->energy)) {
    add_kernel<<<blocks_for(nn2), 256, 0, s>>>(Fd, hd, G, nn2);
    RR_LAUNCH_CHECK();
    if (host) copy_out(F, Fd, nn2, true, s);
  }
  prof_mark(h, 4, s);
  if (host || (o && o->sync)) check_status(h, s);
}

// riFockTwoElectronDirect: G from P_ukb (J) and caller-supplied C_occ_ukb / occupations (K).
void ukb_two_electron(rr_ri_store* h, const double* P, const double* C, int64_t nocc, const double* occ, double* Gout,
                      const rr_opts* o) {
  RR_REQUIRE(h->ntens == 2, RR_ERR_STATE, "rr_ri_two_electron_ukb: needs a 4-component store (rr_ri_create_4c)");
  const int64_t nl = h->n, ns = h->ns, nu = 2 * nl + 2 * ns, nn2 = nu * nu * 2;
  RR_REQUIRE(nocc >= 0 && nocc <= nu, RR_ERR_ARG, "riFockTwoElectronDirect: c_occ_ukb dimension does not match n_ukb x occupations.size()");
  const bool host = !o || o->mem == RR_MEM_HOST;
  cudaStream_t s = call_stream(h, o);
  const int64_t pl = round_up(std::max<int64_t>(nl * nl, 2), 32), ps = round_up(std::max<int64_t>(ns * ns, 2), 32);
  double *DL, *DS, *Ct, *Pd = const_cast<double*>(P), *Cd = const_cast<double*>(C), *od = const_cast<double*>(occ),
         *G = Gout;
  Arena ar(&h->solver_w);
  ar.request(&DL, pl);
  ar.request(&DS, ps);
  ar.request(&Ct, 2 * nu * std::max<int64_t>(nocc, 1));
  if (host) {
    ar.request(&Cd, 2 * nu * std::max<int64_t>(nocc, 1));
    ar.request(&od, nocc);
    ar.request(&Pd, nn2);
    ar.request(&G, nn2);
  }
  ar.commit();
  if (host) {
    copy_in(Pd, P, nn2, true, s);
    copy_in(Cd, C, 2 * nu * nocc, true, s);
    copy_in(od, occ, nocc, true, s);
  }
  prof_mark(h, 0, s);
  RR_CUDA(cudaMemsetAsync(DL, 0, sizeof(double) * pl, s));
  RR_CUDA(cudaMemsetAsync(DS, 0, sizeof(double) * ps, s));
  spin_sum_kernel<<<blocks_for(nl * nl), 256, 0, s>>>(DL, Pd, nu, 0, nl, nl);
  RR_LAUNCH_CHECK();
  if (ns) {
    spin_sum_kernel<<<blocks_for(ns * ns), 256, 0, s>>>(DS, Pd, nu, 2 * nl, 2 * nl + ns, ns);
    RR_LAUNCH_CHECK();
  }
  if (nocc) {
    ct_from_occupied_kernel<<<blocks_for(nocc * nu), 256, 0, s>>>(Ct, Cd, od, nu, nocc);
    RR_LAUNCH_CHECK();
  }
  prof_mark(h, 1, s);
  Flavours fl;
  fl.nf = 4;
  fl.off = {0, nl, 2 * nl, 2 * nl + ns};
  fl.fs = {nl, nl, ns, ns};
  fl.tens = {0, 0, 1, 1};
  const double* dps[2] = {DL, DS};
  two_electron_rel(h, fl, nu, Ct, nocc, dps, G, s, nullptr);
  if (host) copy_out(Gout, G, nn2, true, s);
  prof_mark(h, 4, s);
  if (host || (o && o->sync)) check_status(h, s);
}

// rkbFockMatrix: recovery in the RKB basis with x_full / s_full, embedding with v_total.
// `proj` / `proj_rank` as for fock_x2c (in the orthonormal basis of x_full).
void fock_rkb(rr_ri_store* h, const double* hc, const double* v, int64_t n_rkb, const double* s_full,
              const double* x_full, int64_t n_eff, const double* P, double* F, const rr_opts* o, const RelBuild* rb,
              const double* proj, int64_t proj_rank) {
  RR_REQUIRE(h->ntens == 2, RR_ERR_STATE, "rr_ri_fock_rkb: needs a 4-component store (rr_ri_create_4c)");
  const int64_t nl = h->n, ns = h->ns, nu = 2 * nl + 2 * ns;
  RR_REQUIRE(n_rkb >= 1 && n_eff >= 0 && n_eff <= n_rkb, RR_ERR_ARG, "rr_ri_fock_rkb: bad n_rkb / n_eff");
  const bool host = !o || o->mem == RR_MEM_HOST;
  cudaStream_t s = call_stream(h, o);
  const int64_t rr2 = n_rkb * n_rkb * 2, uu2 = nu * nu * 2, ur2 = nu * n_rkb * 2;
  const int64_t pl = round_up(std::max<int64_t>(nl * nl, 2), 32), ps = round_up(std::max<int64_t>(ns * ns, 2), 32);
  double *DL, *DS, *Ct_rkb, *Ct_ukb, *Pu, *G, *VP, *GV;
  double *hd = const_cast<double*>(hc), *vd = const_cast<double*>(v), *sd = const_cast<double*>(s_full),
         *xd = const_cast<double*>(x_full), *Pd = const_cast<double*>(P), *Fd = F;
  Arena ar(&h->solver_w);
  ar.request(&DL, pl);
  ar.request(&DS, ps);
  ar.request(&Ct_rkb, 2 * n_rkb * std::max<int64_t>(n_eff, 1));
  ar.request(&Ct_ukb, 2 * nu * std::max<int64_t>(n_eff, 1));
  ar.request(&Pu, uu2);
  ar.request(&G, uu2);
  ar.request(&VP, ur2);
  ar.request(&GV, ur2);
  if (host) {
    ar.request(&hd, rr2);
    ar.request(&vd, ur2);
    ar.request(&sd, rr2);
    ar.request(&xd, 2 * n_rkb * n_eff);
    ar.request(&Pd, rr2);
    ar.request(&Fd, rr2);
  }
  ar.commit();
  if (host) {
    copy_in(hd, hc, rr2, true, s);
    copy_in(vd, v, ur2, true, s);
    copy_in(sd, s_full, rr2, true, s);
    copy_in(xd, x_full, 2 * n_rkb * n_eff, true, s);
    copy_in(Pd, P, rr2, true, s);
  }
  prof_mark(h, 0, s);
  int64_t r = proj_rank;
  if (proj) projector_ct(h, proj, nullptr, xd, n_rkb, n_eff, r, true, Ct_rkb, s);
  else r = occupied_ct(h, xd, sd, Pd, n_rkb, n_eff, 1.0, true, true, Ct_rkb, s);
  // c_t (UKB) = c_t (RKB) v_total^dagger  (C_occ_ukb = v_total C_occ_rkb)
  GemmDesc g;
  g.cplx = true;
  if (r > 0) {
    g.M = r; g.N = nu; g.K = n_rkb;
    g.A = Ct_rkb; g.lda = n_rkb; g.B = vd; g.ldb = n_rkb; g.opB = Op::T; g.conjB = true;
    g.C = Ct_ukb; g.ldc = nu;
    gemm(g, s);
  }
  // P_ukb = v P v^dagger, only its four diagonal flavour blocks (all that J reads): each block
  // v_f P v_f^dagger is Hermitian, so upper tiles and a mirror
  GemmDesc a;
  a.cplx = true;
  a.M = nu; a.N = n_rkb; a.K = n_rkb; a.A = vd; a.lda = n_rkb; a.B = Pd; a.ldb = n_rkb; a.C = VP; a.ldc = n_rkb;
  gemm(a, s, h->work.p, static_cast<int64_t>(h->work.n));
  {
    const int64_t boff[4] = {0, nl, 2 * nl, 2 * nl + ns}, bfs[4] = {nl, nl, ns, ns};
    for (int f = 0; f < 4; ++f) {
      if (bfs[f] == 0) continue;
      GemmDesc d;
      d.cplx = true;
      d.M = bfs[f]; d.N = bfs[f]; d.K = n_rkb;
      d.A = VP + 2 * boff[f] * n_rkb; d.lda = n_rkb;
      d.B = vd + 2 * boff[f] * n_rkb; d.ldb = n_rkb; d.opB = Op::T; d.conjB = true;
      d.C = Pu + 2 * (boff[f] * nu + boff[f]); d.ldc = nu;
      d.mirror = 1;
      gemm(d, s, h->work.p, static_cast<int64_t>(h->work.n));
    }
  }
  RR_CUDA(cudaMemsetAsync(DL, 0, sizeof(double) * pl, s));
  RR_CUDA(cudaMemsetAsync(DS, 0, sizeof(double) * ps, s));
  spin_sum_kernel<<<blocks_for(nl * nl), 256, 0, s>>>(DL, Pu, nu, 0, nl, nl);
  RR_LAUNCH_CHECK();
  if (ns) {
    spin_sum_kernel<<<blocks_for(ns * ns), 256, 0, s>>>(DS, Pu, nu, 2 * nl, 2 * nl + ns, ns);
    RR_LAUNCH_CHECK();
  }
  prof_mark(h, 1, s);
  Flavours fl;
  fl.nf = 4;
  fl.off = {0, nl, 2 * nl, 2 * nl + ns};
  fl.fs = {nl, nl, ns, ns};
  fl.tens = {0, 0, 1, 1};
  const double* dps[2] = {DL, DS};
  two_electron_rel(h, fl, nu, Ct_ukb, r, dps, G, s, rb);
  if (rb && rb->energy) {  // energy-only evaluation: no F
    prof_mark(h, 4, s);
    if (host || (o && o->sync)) check_status(h, s);
    return;
  }
  // F = h + v^dagger G v
  GemmDesc b;
  b.cplx = true;
  b.M = nu; b.N = n_rkb; b.K = nu; b.A = G; b.lda = nu; b.B = vd; b.ldb = n_rkb; b.C = GV; b.ldc = n_rkb;
  gemm(b, s);
  if (Fd != hd) copy_out(Fd, hd, rr2, false, s);
  b.M = n_rkb; b.N = n_rkb; b.K = nu; b.A = vd; b.lda = n_rkb; b.opA = Op::T; b.conjA = true; b.B = GV; b.ldb = n_rkb;
  b.C = Fd; b.ldc = n_rkb; b.beta = 1.0;
  b.mirror = 1;  // F = h + v^dagger G v is Hermitian
  gemm(b, s, h->work.p, static_cast<int64_t>(h->work.n));
  if (host) copy_out(F, Fd, rr2, true, s);
  prof_mark(h, 4, s);
  if (host || (o && o->sync)) check_status(h, s);
}

}  // namespace rr
