// MO-basis RI tensors and their consumers (the functional stage's hot path).
//
// References:
//   buildRiNonRelSpinMoEri / rotated / embeddedB / operator()   src/NON_REL/NonRelSpinRiMoEri.cpp:13-95, .h:40-89
//   buildRiMoEri (+ transformBlock) / rotated / positiveBlock    src/UKB/RiMoEri.cpp:20-120
//   RiMoEri::operator() (J_ij, K_ij, L_ij reads)                 src/UKB/RiMoEri.h:50-57, src/Occ_opt/PNOFs.cpp:306-321
//   riHxFockGemm (generalized Fock)                              src/Hessian_opt/RiGemmFock.cpp:52-157
//
// A rr_mo_store keeps the MO tensor resident: (naux, n*n) real for the nonrelativistic spin-orbital
// kind (n = spatial orbitals; the spin-orbital accessors have dimension 2n and the reference's spin
// selection rule), or (naux, n*n) complex interleaved for the relativistic kind.  Every contraction
// runs on the FP64 DMMA GEMM family; the transforms are chunked over the aux index so that the
// per-chunk intermediate stays within ~64 MB.
#include <algorithm>
#include <cmath>
#include <vector>

#include "mo_store.cuh"

namespace rr {

namespace {

int blocks_for(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 2368))); }

// A_f (2 nt x fs, real) = [Re(c_block)^T ; -Im(c_block)^T] for rows [off, off+fs) of c_ukb (complex
// n_ukb x nt): the stacked real form of c_block^dagger.
__global__ void cdag_stack_kernel(double* A, const double* c, int64_t nt, int64_t off, int64_t fs) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < 2 * nt * fs;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = idx / fs, a = idx % fs;
    const int64_t p = r < nt ? r : r - nt;
    const double* z = c + ((off + a) * nt + p) * 2;
    A[idx] = r < nt ? z[0] : -z[1];
  }
}

// out[P][s] = B[P][s*n + s]  (PL = 1 real, 2 complex)
template <int PL>
__global__ void diag_gather_kernel(double* out, const double* B, int64_t naux, int64_t n) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < naux * n;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t P = idx / n, s = idx % n;
    for (int q = 0; q < PL; ++q) out[idx * PL + q] = B[(P * n * n + s * n + s) * PL + q];
  }
}

// K[a][b] = sum_P B[P][a][b] * B[P][b][a] (complex product, no conjugation), 32x32 tiles with the
// mirrored tile staged through shared memory so both reads are coalesced.  Deterministic.
template <int PL>
__global__ void kmat_kernel(const double* B, int64_t naux, int64_t n, double* K) {
  __shared__ double tt[32][33 * PL];
  const int64_t i0 = static_cast<int64_t>(blockIdx.y) * 32, j0 = static_cast<int64_t>(blockIdx.x) * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  double ar[4] = {0, 0, 0, 0}, ai[4] = {0, 0, 0, 0};
  for (int64_t P = 0; P < naux; ++P) {
    const double* b = B + P * n * n * PL;
    // stage tile B[j0.., i0..] (rows j, cols i) transposed
    for (int r = ty; r < 32; r += 8) {
      const int64_t j = j0 + r, i = i0 + tx;
      for (int q = 0; q < PL; ++q) tt[r][tx * PL + q] = (j < n && i < n) ? b[(j * n + i) * PL + q] : 0.0;
    }
    __syncthreads();
    for (int k = 0; k < 4; ++k) {
      const int r = ty + 8 * k;
      const int64_t i = i0 + r, j = j0 + tx;
      if (i < n && j < n) {
        const double xr = b[(i * n + j) * PL], xi = PL == 2 ? b[(i * n + j) * PL + 1] : 0.0;
        const double yr = tt[tx][r * PL], yi = PL == 2 ? tt[tx][r * PL + 1] : 0.0;  // B[j][i]
        ar[k] += xr * yr - xi * yi;
        if (PL == 2) ai[k] += xr * yi + xi * yr;
      }
    }
    __syncthreads();
  }
  for (int k = 0; k < 4; ++k) {
    const int64_t i = i0 + ty + 8 * k, j = j0 + tx;
    if (i < n && j < n) {
      K[(i * n + j) * PL] = ar[k];
      if (PL == 2) K[(i * n + j) * PL + 1] = ai[k];
    }
  }
}

// Nonrelativistic spin-orbital expansion of spatial J/K (n x n) to 2n x 2n with the spin selection
// rule of src/NON_REL/NonRelSpinRiMoEri.h:40 (eri(A,B,C,D) = 0 unless spin(A)=spin(C), spin(B)=spin(D)):
//   J2(i,j) = eri(i,j,i,j) = J(i%n, j%n);  K2(i,j) = eri(i,j,j,i) = [spin i == spin j] K(i%n, j%n).
__global__ void spin_expand_kernel(const double* J, const double* K, int64_t n, double* J2, double* K2) {
  const int64_t m = 2 * n;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < m * m;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx / m, j = idx % m;
    const int64_t si = i % n, sj = j % n;
    J2[idx] = J[si * n + sj];
    K2[idx] = (i / n == j / n) ? K[si * n + sj] : 0.0;
  }
}

// L(i,j) = eri(pbar_i, j, j, pbar_i) = Kfull(pbar_i, j) (K as produced above; PL interleave).
template <int PL>
__global__ void l_from_k_kernel(const double* K, const int64_t* pair_of, int64_t m, double* L) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < m * m;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx / m, j = idx % m;
    const int64_t pb = pair_of[i];
    for (int q = 0; q < PL; ++q) L[idx * PL + q] = K[(pb * m + j) * PL + q];
  }
}

// Batched element access eri(a,b,c,d) = sum_P B(P, a, c) B(P, b, d) over the stored indices
// (already mapped: for the nonrelativistic kind the spin selection is applied by the caller).
template <int PL>
__global__ void eri_elements_kernel(const double* B, int64_t naux, int64_t n, const int64_t* quads, int64_t count,
                                    int spin_n, double* out) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= count) return;
  int64_t a = quads[4 * warp], b = quads[4 * warp + 1], c = quads[4 * warp + 2], d = quads[4 * warp + 3];
  bool zero = false;
  if (spin_n > 0) {
    zero = (a / spin_n != c / spin_n) || (b / spin_n != d / spin_n);
    a %= spin_n; b %= spin_n; c %= spin_n; d %= spin_n;
  }
  double sr = 0.0, si = 0.0;
  if (!zero) {
    const int64_t ac = a * n + c, bd = b * n + d;
    for (int64_t P = lane; P < naux; P += 32) {
      const double* bp = B + P * n * n * PL;
      const double xr = bp[ac * PL], xi = PL == 2 ? bp[ac * PL + 1] : 0.0;
      const double yr = bp[bd * PL], yi = PL == 2 ? bp[bd * PL + 1] : 0.0;
      sr += xr * yr - xi * yi;
      si += xr * yi + xi * yr;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    sr += __shfl_xor_sync(0xffffffffu, sr, o);
    si += __shfl_xor_sync(0xffffffffu, si, o);
  }
  if (lane == 0) {
    out[warp * PL] = sr;
    if (PL == 2) out[warp * PL + 1] = si;
  }
}

// out[P] (m x m) = B[P] (n x n) restricted to [off, n) on both legs.
template <int PL>
__global__ void subblock_kernel(double* out, const double* B, int64_t naux, int64_t n, int64_t off) {
  const int64_t m = n - off;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < naux * m * m;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t P = idx / (m * m), r = idx % (m * m), a = r / m, c = r % m;
    for (int q = 0; q < PL; ++q) out[idx * PL + q] = B[(P * n * n + (a + off) * n + c + off) * PL + q];
  }
}

// Block-diagonal (alpha, beta) embedding of a spatial tensor (src/NON_REL/NonRelSpinRiMoEri.h:77).
__global__ void embed_kernel(double* out, const double* B, int64_t naux, int64_t n) {
  const int64_t m = 2 * n;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < naux * m * m;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t P = idx / (m * m), r = idx % (m * m), i = r / m, j = r % m;
    out[idx] = (i / n == j / n) ? B[P * n * n + (i % n) * n + (j % n)] : 0.0;
  }
}

// u = (U_aa + U_bb)/2 of a 2n x 2n spin-orbital rotation (src/NON_REL/NonRelSpinRiMoEri.cpp:191-193),
// and dev[0] = max |off-diagonal blocks|, dev[1] = max |U_bb - U_aa| (zeroed by the caller).
__global__ void spin_average_kernel(const double* U, int64_t n, double* u, double* dev) {
  double m0 = 0.0, m1 = 0.0;
  const int64_t m = 2 * n;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < n * n;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx / n, j = idx % n;
    const double aa = U[i * m + j], bb = U[(n + i) * m + n + j];
    u[idx] = 0.5 * (aa + bb);
    m0 = fmax(m0, fmax(fabs(U[i * m + n + j]), fabs(U[(n + i) * m + j])));
    m1 = fmax(m1, fabs(bb - aa));
  }
  for (int o = 16; o > 0; o >>= 1) {
    m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, o));
    m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(reinterpret_cast<unsigned long long*>(dev), static_cast<unsigned long long>(__double_as_longlong(m0)));
    atomicMax(reinterpret_cast<unsigned long long*>(dev + 1), static_cast<unsigned long long>(__double_as_longlong(m1)));
  }
}

// Generalized-Fock pieces (src/Hessian_opt/RiGemmFock.cpp:92-157).
// F(p,q) = occ_q h(q,p) + sum_P B(P,q,p) W(P,q)
template <int PL>
__global__ void hx_f0f1_kernel(const double* B, const double* W, const double* h, const double* occ, int64_t naux,
                               int64_t n, double* F) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < n * n;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t q = idx / n, p = idx % n;  // p fastest: B(P,q,p) reads coalesced
    double sr = 0.0, si = 0.0;
    for (int64_t P = 0; P < naux; ++P) {
      const double br = B[(P * n * n + q * n + p) * PL], bi = PL == 2 ? B[(P * n * n + q * n + p) * PL + 1] : 0.0;
      const double wr = W[(P * n + q) * PL], wi = PL == 2 ? W[(P * n + q) * PL + 1] : 0.0;
      sr += br * wr - bi * wi;
      si += br * wi + bi * wr;
    }
    const double o = occ[q];
    double* f = F + (p * n + q) * PL;
    f[0] = o * h[(q * n + p) * PL] + sr;
    if (PL == 2) f[1] = o * h[(q * n + p) * PL + 1] + si;
  }
}

// Y(P,t,q) = -x2(q,t) B(P,q,t) [+ 2 (l1(st,qbar) + l2(st,q)) B(P,st,qbar), st = pair_of[t]] for a
// chunk of aux rows [P0, P0 + pc).
template <int PL>
__global__ void hx_y_kernel(const double* B, int64_t P0, int64_t pc, int64_t n, const double* x2, const int64_t* pair_of,
                            const double* l1, const double* l2, double* Y) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < pc * n * n;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t pl = idx / (n * n), r = idx % (n * n), t = r / n, q = r % n;
    const double* bp = B + (P0 + pl) * n * n * PL;
    const double c = -x2[q * n + t];
    double vr = c * bp[(q * n + t) * PL];
    double vi = PL == 2 ? c * bp[(q * n + t) * PL + 1] : 0.0;
    if (pair_of) {
      const int64_t st = pair_of[t], qb = pair_of[q];
      const double w = 2.0 * (l1[st * n + qb] + l2[st * n + q]);
      vr += w * bp[(st * n + qb) * PL];
      if (PL == 2) vi += w * bp[(st * n + qb) * PL + 1];
    }
    Y[idx * PL] = vr;
    if (PL == 2) Y[idx * PL + 1] = vi;
  }
}

__global__ void real_to_complex_kernel(double* out, const double* in, int64_t count) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    out[2 * i] = in[i];
    out[2 * i + 1] = 0.0;
  }
}

__global__ void add_inplace_kernel(double* y, const double* x, int64_t count) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    y[i] += x[i];
}

int64_t chunk_rows(int64_t naux, int64_t per_row_doubles) {
  const int64_t budget = 8 * 1024 * 1024;  // doubles (64 MB) per chunk intermediate
  return std::max<int64_t>(1, std::min<int64_t>(naux, budget / std::max<int64_t>(per_row_doubles, 1)));
}

}  // namespace

cudaStream_t mo_stream(rr_mo_store* m, const rr_opts* o) {
  if (o && o->stream) return static_cast<cudaStream_t>(o->stream);
  return m->ctx.main;
}

// ---------------------------------------------------------------- builds

// B_mo^P = C^T B^P C (real, n x n), chunked over P: T = C^T B^P, then T C.
void mo_build_nonrel(rr_ri_store* ri, const double* C, rr_mo_store* m, bool host, cudaStream_t s) {
  const int64_t n = ri->n, naux = ri->naux;
  m->B.ensure(static_cast<size_t>(std::max<int64_t>(naux * n * n, 1)));  // a rebuild keeps the tensor's memory
  m->scratch.ensure(static_cast<size_t>(round_up(n * n, 32)));
  double* Cd = m->scratch.p;
  copy_in(Cd, C, n * n, host, s);
  const int64_t pc = chunk_rows(naux, n * n);
  m->T.ensure(static_cast<size_t>(pc * n * n));
  for (int64_t P0 = 0; P0 < naux; P0 += pc) {
    const int64_t cnt = std::min(pc, naux - P0);
    GemmDesc a;  // T[P] = C^T B^P
    a.M = n; a.N = n; a.K = n;
    a.A = Cd; a.lda = n; a.opA = Op::T;
    a.B = ri->B[0].p + P0 * ri->pitch[0]; a.ldb = n; a.strideB = ri->pitch[0];
    a.C = m->T.p; a.ldc = n; a.strideC = n * n;
    a.batch = cnt;
    gemm(a, s);
    GemmDesc b;  // B_mo[P] = T[P] C
    b.M = n; b.N = n; b.K = n;
    b.A = m->T.p; b.lda = n; b.strideA = n * n;
    b.B = Cd; b.ldb = n;
    b.C = m->B.p + P0 * n * n; b.ldc = n; b.strideC = n * n;
    b.batch = cnt;
    gemm(b, s);
  }
}

// buildRiMoEri: B_mo^P = sum over the four UKB blocks of c_f^dagger B_f^P c_f (complex nt x nt).
void mo_build_ukb(rr_ri_store* ri, const double* c_ukb, int64_t nt, rr_mo_store* m, bool host, cudaStream_t s) {
  const int64_t nl = ri->n, ns = ri->ns, naux = ri->naux, nu = 2 * nl + 2 * ns;
  const int64_t off[4] = {0, nl, 2 * nl, 2 * nl + ns}, fs[4] = {nl, nl, ns, ns};
  const int tens[4] = {0, 0, 1, 1};
  m->B.alloc(static_cast<size_t>(std::max<int64_t>(2 * naux * nt * nt, 1)));
  const int64_t fsmax = std::max(nl, ns);
  m->scratch.ensure(static_cast<size_t>(round_up(2 * nu * nt, 32) + round_up(2 * nt * fsmax, 32)));
  double* cd = m->scratch.p;
  double* Af = m->scratch.p + round_up(2 * nu * nt, 32);
  copy_in(cd, c_ukb, 2 * nu * nt, host, s);
  const int64_t pc = chunk_rows(naux, 2 * nt * fsmax);
  m->T.ensure(static_cast<size_t>(pc * 2 * nt * fsmax));
  bool first = true;
  for (int f = 0; f < 4; ++f) {
    if (fs[f] == 0 || nt == 0) continue;
    cdag_stack_kernel<<<blocks_for(2 * nt * fs[f]), 256, 0, s>>>(Af, cd, nt, off[f], fs[f]);
    RR_LAUNCH_CHECK();
    for (int64_t P0 = 0; P0 < naux; P0 += pc) {
      const int64_t cnt = std::min(pc, naux - P0);
      GemmDesc a;  // T[P] = c_f^dagger B_f^P  (stacked real rows -> interleaved complex nt x fs)
      a.M = 2 * nt; a.N = fs[f]; a.K = fs[f];
      a.A = Af; a.lda = fs[f];
      a.B = ri->B[tens[f]].p + P0 * ri->pitch[tens[f]]; a.ldb = fs[f]; a.strideB = ri->pitch[tens[f]];
      a.C = m->T.p; a.ldc = 2 * fs[f]; a.strideC = 2 * nt * fs[f];
      a.c_plane_rows = nt; a.c_plane_stride = 1; a.c_col_stride = 2;
      a.batch = cnt;
      gemm(a, s);
      GemmDesc b;  // B_mo[P] (+)= T[P] c_f
      b.cplx = true;
      b.M = nt; b.N = nt; b.K = fs[f];
      b.A = m->T.p; b.lda = fs[f]; b.strideA = nt * fs[f];
      b.B = cd + off[f] * nt * 2; b.ldb = nt;
      b.C = m->B.p + 2 * P0 * nt * nt; b.ldc = nt; b.strideC = nt * nt;
      b.beta = first ? 0.0 : 1.0;
      b.batch = cnt;
      gemm(b, s);
    }
    first = false;
  }
  if (first) RR_CUDA(cudaMemsetAsync(m->B.p, 0, sizeof(double) * m->B.n, s));
}

// ---------------------------------------------------------------- rotations and views

// Real: B' = u^T B u with u the alpha/beta-averaged spatial block; complex: B' = U^dagger B U.
void mo_rotate(rr_mo_store* src, const double* U, rr_mo_store* dst, bool host, cudaStream_t s) {
  const int64_t n = src->n, naux = src->naux;
  const int PL = src->cplx ? 2 : 1;
  dst->B.alloc(static_cast<size_t>(std::max<int64_t>(PL * naux * n * n, 1)));
  const int64_t ulen = src->cplx ? 2 * n * n : 4 * n * n;
  src->scratch.ensure(static_cast<size_t>(round_up(ulen, 32) + round_up(PL * n * n, 32) + 32));
  double* Ud = src->scratch.p;
  double* u = src->scratch.p + round_up(ulen, 32);
  double* dev = u + round_up(PL * n * n, 32);
  copy_in(Ud, U, ulen, host, s);
  if (!src->cplx) {
    RR_CUDA(cudaMemsetAsync(dev, 0, 2 * sizeof(double), s));
    spin_average_kernel<<<blocks_for(n * n), 256, 0, s>>>(Ud, n, u, dev);
    RR_LAUNCH_CHECK();
    double hd[2];
    RR_CUDA(cudaMemcpyAsync(hd, dev, sizeof(hd), cudaMemcpyDeviceToHost, s));
    RR_CUDA(cudaStreamSynchronize(s));
    if (hd[0] > 1e-3 || hd[1] > 1e-3)
      throw Error(RR_ERR_ARG, "RiNonRelSpinMoEri::rotated: rotation is not spin-restricted (alpha and beta rotations differ by " +
                                  std::to_string(hd[1]) + ", cross-spin block max " + std::to_string(hd[0]) + ")");
  } else {
    u = Ud;
  }
  const int64_t pc = chunk_rows(naux, PL * n * n);
  src->T.ensure(static_cast<size_t>(pc * PL * n * n));
  for (int64_t P0 = 0; P0 < naux; P0 += pc) {
    const int64_t cnt = std::min(pc, naux - P0);
    GemmDesc a;  // T = u^dagger B^P
    a.cplx = src->cplx;
    a.M = n; a.N = n; a.K = n;
    a.A = u; a.lda = n; a.opA = Op::T; a.conjA = src->cplx;
    a.B = src->B.p + PL * P0 * n * n; a.ldb = n; a.strideB = n * n;
    a.C = src->T.p; a.ldc = n; a.strideC = n * n;
    a.batch = cnt;
    gemm(a, s);
    GemmDesc b;  // B' = T u
    b.cplx = src->cplx;
    b.M = n; b.N = n; b.K = n;
    b.A = src->T.p; b.lda = n; b.strideA = n * n;
    b.B = u; b.ldb = n;
    b.C = dst->B.p + PL * P0 * n * n; b.ldc = n; b.strideC = n * n;
    b.batch = cnt;
    gemm(b, s);
  }
}

void mo_positive_block(rr_mo_store* src, int64_t off, rr_mo_store* dst, cudaStream_t s) {
  const int64_t m = src->n - off, naux = src->naux;
  const int PL = src->cplx ? 2 : 1;
  dst->B.alloc(static_cast<size_t>(std::max<int64_t>(PL * naux * m * m, 1)));
  if (naux * m * m == 0) return;
  if (PL == 2) subblock_kernel<2><<<blocks_for(naux * m * m), 256, 0, s>>>(dst->B.p, src->B.p, naux, src->n, off);
  else subblock_kernel<1><<<blocks_for(naux * m * m), 256, 0, s>>>(dst->B.p, src->B.p, naux, src->n, off);
  RR_LAUNCH_CHECK();
}

const double* mo_operand(rr_mo_store* m, cudaStream_t s, int64_t* d) {
  if (m->cplx) {
    *d = m->n;
    return m->B.p;
  }
  const int64_t dd = 4 * m->n * m->n;
  *d = 2 * m->n;
  m->emb.ensure(static_cast<size_t>(std::max<int64_t>(m->naux * dd, 1)));
  if (m->naux * dd) {
    embed_kernel<<<blocks_for(m->naux * dd), 256, 0, s>>>(m->emb.p, m->B.p, m->naux, m->n);
    RR_LAUNCH_CHECK();
  }
  return m->emb.p;
}

void mo_embedded(rr_mo_store* m, double* out, bool host, cudaStream_t s) {
  const int64_t n = m->n, naux = m->naux, cnt = naux * 4 * n * n;
  double* dst = out;
  if (host) {
    m->T.ensure(static_cast<size_t>(std::max<int64_t>(cnt, 1)));
    dst = m->T.p;
  }
  if (cnt) {
    embed_kernel<<<blocks_for(cnt), 256, 0, s>>>(dst, m->B.p, naux, n);
    RR_LAUNCH_CHECK();
  }
  if (host) copy_out(out, dst, cnt, true, s);
}

// ---------------------------------------------------------------- element access and J/K/L

void mo_eri(rr_mo_store* m, int64_t count, const int64_t* quads, double* out, bool host, cudaStream_t s) {
  const int PL = m->cplx ? 2 : 1;
  if (count == 0) return;
  m->scratch.ensure(static_cast<size_t>(round_up(4 * count, 32) + round_up(PL * count, 32)));
  int64_t* q = reinterpret_cast<int64_t*>(m->scratch.p);
  double* o = m->scratch.p + round_up(4 * count, 32);
  if (host) RR_CUDA(cudaMemcpyAsync(q, quads, sizeof(int64_t) * 4 * count, cudaMemcpyHostToDevice, s));
  else q = const_cast<int64_t*>(quads);
  if (!host) o = out;
  const int64_t threads = count * 32;
  const int spin_n = m->cplx ? 0 : static_cast<int>(m->n);
  if (PL == 2) eri_elements_kernel<2><<<ceil_div(threads, 256), 256, 0, s>>>(m->B.p, m->naux, m->n, q, count, spin_n, o);
  else eri_elements_kernel<1><<<ceil_div(threads, 256), 256, 0, s>>>(m->B.p, m->naux, m->n, q, count, spin_n, o);
  RR_LAUNCH_CHECK();
  if (host) copy_out(out, o, PL * count, true, s);
}

// J_ij = eri(i,j,i,j), K_ij = eri(i,j,j,i), L_ij = eri(pbar_i, j, j, pbar_i) over the accessor's
// dimension (2n for the nonrelativistic spin-orbital kind, n_total for the complex kind).
void mo_jkl(rr_mo_store* m, const int64_t* pair_of, double* J, double* K, double* L, bool host, cudaStream_t s) {
  const int64_t n = m->n, naux = m->naux;
  const int PL = m->cplx ? 2 : 1;
  const int64_t dim = m->cplx ? n : 2 * n;
  const int64_t out_sz = PL * dim * dim;
  m->scratch.ensure(static_cast<size_t>(round_up(PL * naux * n, 32) + 2 * round_up(PL * n * n, 32) + 3 * round_up(out_sz, 32) +
                                        round_up(dim, 32) + 64));
  double* bd = m->scratch.p;
  double* Jn = bd + round_up(PL * naux * n, 32);
  double* Kn = Jn + round_up(PL * n * n, 32);
  double* Jo = Kn + round_up(PL * n * n, 32);
  double* Ko = Jo + round_up(out_sz, 32);
  double* Lo = Ko + round_up(out_sz, 32);
  int64_t* po = reinterpret_cast<int64_t*>(Lo + round_up(out_sz, 32));
  if (PL == 2) diag_gather_kernel<2><<<blocks_for(naux * n), 256, 0, s>>>(bd, m->B.p, naux, n);
  else diag_gather_kernel<1><<<blocks_for(naux * n), 256, 0, s>>>(bd, m->B.p, naux, n);
  RR_LAUNCH_CHECK();
  GemmDesc g;  // J = Bd^T Bd (no conjugation)
  g.cplx = m->cplx;
  g.M = n; g.N = n; g.K = naux;
  g.A = bd; g.lda = n; g.opA = Op::T;
  g.B = bd; g.ldb = n; g.C = Jn; g.ldc = n;
  m->work.ensure(static_cast<size_t>(std::max<int64_t>(gemm_work_doubles(g), 1)));
  gemm(g, s, m->work.p, static_cast<int64_t>(m->work.n));
  dim3 grid(ceil_div(n, 32), ceil_div(n, 32)), blk(32, 8);
  if (n > 0 && naux > 0) {
    if (PL == 2) kmat_kernel<2><<<grid, blk, 0, s>>>(m->B.p, naux, n, Kn);
    else kmat_kernel<1><<<grid, blk, 0, s>>>(m->B.p, naux, n, Kn);
    RR_LAUNCH_CHECK();
  } else {
    RR_CUDA(cudaMemsetAsync(Kn, 0, sizeof(double) * PL * n * n, s));
  }
  if (m->cplx) {
    copy_out(Jo, Jn, out_sz, false, s);
    copy_out(Ko, Kn, out_sz, false, s);
  } else {
    spin_expand_kernel<<<blocks_for(dim * dim), 256, 0, s>>>(Jn, Kn, n, Jo, Ko);
    RR_LAUNCH_CHECK();
  }
  if (L && pair_of) {
    if (host) RR_CUDA(cudaMemcpyAsync(po, pair_of, sizeof(int64_t) * dim, cudaMemcpyHostToDevice, s));
    else RR_CUDA(cudaMemcpyAsync(po, pair_of, sizeof(int64_t) * dim, cudaMemcpyDeviceToDevice, s));
    if (PL == 2) l_from_k_kernel<2><<<blocks_for(dim * dim), 256, 0, s>>>(Ko, po, dim, Lo);
    else l_from_k_kernel<1><<<blocks_for(dim * dim), 256, 0, s>>>(Ko, po, dim, Lo);
    RR_LAUNCH_CHECK();
    copy_out(L, Lo, out_sz, host, s);
  }
  copy_out(J, Jo, out_sz, host, s);
  copy_out(K, Ko, out_sz, host, s);
}

// ---------------------------------------------------------------- generalized Fock

// riHxFockGemm on a tensor Bt (naux, d*d) of element kind PL.  All matrix arguments on the device.
void hx_fock_core(rr_mo_store* m, const double* Bt, int64_t d, int PL, const double* h, const double* occ,
                  const double* h2, const double* x2, const int64_t* pair_of, const double* l1, const double* l2,
                  double* F, cudaStream_t s) {
  const int64_t naux = m->naux;
  const bool cplx = PL == 2;
  Arena ar(&m->hx);
  double *bd, *h2c, *W, *G;
  ar.request(&bd, PL * naux * d);
  ar.request(&h2c, PL * d * d);
  ar.request(&W, PL * naux * d);
  ar.request(&G, PL * d * d);
  ar.commit();
  if (d == 0) return;
  if (cplx) diag_gather_kernel<2><<<blocks_for(naux * d), 256, 0, s>>>(bd, Bt, naux, d);
  else diag_gather_kernel<1><<<blocks_for(naux * d), 256, 0, s>>>(bd, Bt, naux, d);
  RR_LAUNCH_CHECK();
  const double* h2use = h2;
  if (cplx) {
    real_to_complex_kernel<<<blocks_for(d * d), 256, 0, s>>>(h2c, h2, d * d);
    RR_LAUNCH_CHECK();
    h2use = h2c;
  }
  GemmDesc w;  // W = Bdiag h2
  w.cplx = cplx;
  w.M = naux; w.N = d; w.K = d;
  w.A = bd; w.lda = d; w.B = h2use; w.ldb = d; w.C = W; w.ldc = d;
  gemm(w, s);
  if (cplx) hx_f0f1_kernel<2><<<blocks_for(d * d), 256, 0, s>>>(Bt, W, h, occ, naux, d, F);
  else hx_f0f1_kernel<1><<<blocks_for(d * d), 256, 0, s>>>(Bt, W, h, occ, naux, d, F);
  RR_LAUNCH_CHECK();
  // G = sum over aux chunks of B_view^T Y, B_view = (pc*d) x d rows (P,t), Y likewise
  const int64_t pc = chunk_rows(naux, PL * d * d);
  m->T.ensure(static_cast<size_t>(std::max<int64_t>(pc * PL * d * d, 1)));
  bool first = true;
  for (int64_t P0 = 0; P0 < naux; P0 += pc) {
    const int64_t cnt = std::min(pc, naux - P0);
    if (cplx) hx_y_kernel<2><<<blocks_for(cnt * d * d), 256, 0, s>>>(Bt, P0, cnt, d, x2, pair_of, l1, l2, m->T.p);
    else hx_y_kernel<1><<<blocks_for(cnt * d * d), 256, 0, s>>>(Bt, P0, cnt, d, x2, pair_of, l1, l2, m->T.p);
    RR_LAUNCH_CHECK();
    GemmDesc g;
    g.cplx = cplx;
    g.M = d; g.N = d; g.K = cnt * d;
    g.A = Bt + PL * P0 * d * d; g.lda = d; g.opA = Op::T;
    g.B = m->T.p; g.ldb = d;
    g.C = G; g.ldc = d;
    g.beta = first ? 0.0 : 1.0;
    m->work.ensure(static_cast<size_t>(std::max<int64_t>(gemm_work_doubles(g), 1)));
    gemm(g, s, m->work.p, static_cast<int64_t>(m->work.n));
    first = false;
  }
  if (!first) {
    add_inplace_kernel<<<blocks_for(PL * d * d), 256, 0, s>>>(F, G, PL * d * d);
    RR_LAUNCH_CHECK();
  }
}

void mo_hx_fock(rr_mo_store* m, const double* h, const double* occ, const double* h2, const double* x2,
                const int64_t* pair_of, const double* l1, const double* l2, double* F, bool host, cudaStream_t s) {
  const int PL = m->cplx ? 2 : 1;
  const int64_t d = m->cplx ? m->n : 2 * m->n;  // the nonrelativistic overload works on embeddedB (2n)
  const int64_t dd = d * d;
  Arena ar(&m->io);
  double *hd, *od, *h2d, *x2d, *l1d = nullptr, *l2d = nullptr, *Fd, *emb = nullptr, *po_buf = nullptr;
  ar.request(&hd, PL * dd);
  ar.request(&od, d);
  ar.request(&h2d, dd);
  ar.request(&x2d, dd);
  ar.request(&Fd, PL * dd);
  if (pair_of) {
    ar.request(&l1d, dd);
    ar.request(&l2d, dd);
    ar.request(&po_buf, d);  // int64 pair map (8 bytes per entry, like a double)
  }
  ar.commit();
  int64_t* pod = reinterpret_cast<int64_t*>(po_buf);
  auto in = [&](double* dst, const double* src, int64_t cnt) { copy_in(dst, src, cnt, host, s); };
  in(hd, h, PL * dd);
  in(od, occ, d);
  in(h2d, h2, dd);
  in(x2d, x2, dd);
  if (pair_of) {
    in(l1d, l1, dd);
    in(l2d, l2, dd);
    RR_CUDA(cudaMemcpyAsync(pod, pair_of, sizeof(int64_t) * d, host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
  }
  const double* Bt = m->B.p;
  if (!m->cplx) {
    m->emb.ensure(static_cast<size_t>(std::max<int64_t>(m->naux * dd, 1)));
    emb = m->emb.p;
    if (m->naux * dd) {
      embed_kernel<<<blocks_for(m->naux * dd), 256, 0, s>>>(emb, m->B.p, m->naux, m->n);
      RR_LAUNCH_CHECK();
    }
    Bt = emb;
  }
  hx_fock_core(m, Bt, d, PL, hd, od, h2d, x2d, pair_of ? pod : nullptr, l1d, l2d, Fd, s);
  copy_out(F, Fd, PL * dd, host, s);
}

}  // namespace rr
