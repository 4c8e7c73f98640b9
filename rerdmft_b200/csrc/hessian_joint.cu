// hartreeExchangeJointHessianDiagonal on a complex RI MO tensor (the RiMoEri instantiation,
// src/Hessian_opt/HartreeExchangeHessian.cpp:653-711): per rotation pair (p, q) the diagonal of the joint
// [real; imaginary] orbital Hessian,
//   d[I]          =  Re(G_pq,pq - G_pq,qp - G_qp,pq + G_qp,qp),
//   d[npairs + I] = -Re(G_pq,pq + G_pq,qp + G_qp,pq + G_qp,qp),
// with G the bare H/X term (:57-99) plus the L1/L2 pair term (:124-161).  The labels of the learned
// preconditioner for complex (X2C / 4c) orbitals.
//
// With eri(a,b,c,d) = sum_P B(P,a,c) B(P,b,d) (unconjugated, RiMoEri::operator()) and p != q, the four bare
// H/X terms need only J(a,b) = eri(a,b,a,b), K(a,b) = eri(a,b,b,a), Q(a,b) = eri(a,a,b,b) = sum_P B(P,a,b)^2
// and M(a,b) = sum_u two_rdm_h(a,u) (K(u,b) - J(u,b)): the delta sums collapse onto M, the two leftover
// integrals onto J, K or Q.  The pair terms evaluate their integrals directly (one warp per pair).
#include <algorithm>

#include "mo_store.cuh"

namespace rr {
namespace {

int blocks_for(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4736))); }

struct Cx {
  double re, im;
};
__device__ __forceinline__ Cx cx(double r, double i = 0.0) { return {r, i}; }
__device__ __forceinline__ Cx operator+(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ Cx operator-(Cx a, Cx b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ Cx operator*(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ Cx operator*(Cx a, double s) { return {a.re * s, a.im * s}; }
__device__ __forceinline__ Cx conjc(Cx a) { return {a.re, -a.im}; }

struct JointArgs {
  const double* H;  // complex n x n
  const double* F;  // complex n x n (hartreeExchangeFockMatrix's F; ftex(a, b) = F(b, a))
  const double* occ;
  const double* h2;  // real n x n
  const double* x2;
  const double* J;  // complex n x n
  const double* K;
  const double* Q;
  const double* M;
  const double* B;  // complex naux x n^2 (pair terms)
  const int64_t* pairs;  // npairs x 2 (p, q)
  const int64_t* po;     // pair_of or null
  const double* l1;
  const double* l2;
  int64_t n, naux, npairs;
  double* out;
};

__device__ __forceinline__ Cx at(const double* m, int64_t n, int64_t i, int64_t j) {
  return cx(m[2 * (i * n + j)], m[2 * (i * n + j) + 1]);
}

// eri(a,b,c,d) = sum_P B(P,a,c) B(P,b,d), summed by one warp (every lane returns the total).
__device__ Cx eri_warp(const JointArgs& A, int64_t a, int64_t b, int64_t c, int64_t d) {
  const int lane = threadIdx.x & 31;
  const int64_t n2 = A.n * A.n;
  double re = 0.0, im = 0.0;
  for (int64_t P = lane; P < A.naux; P += 32) {
    const Cx x = at(A.B + 2 * P * n2, A.n, a, c), y = at(A.B + 2 * P * n2, A.n, b, d);
    const Cx z = x * y;
    re += z.re;
    im += z.im;
  }
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
  }
  return cx(re, im);
}

// Bare L1/L2 term of G_pq,rs (HartreeExchangeHessian.cpp:124-161), complex, one warp.
__device__ Cx raw_l(const JointArgs& A, int64_t p, int64_t q, int64_t r, int64_t s) {
  const int64_t* po = A.po;
  const int64_t n = A.n;
  Cx t = cx(0.0);
  if (q == po[s]) {
    Cx sum = cx(0.0);
    for (int64_t u = 0; u < n; ++u) sum = sum + eri_warp(A, u, po[u], p, r) * (A.l1[u * n + s] + A.l2[u * n + q]);
    t = t - sum * 2.0;
  }
  {
    const double c = A.l1[r * n + q] + A.l2[r * n + po[q]];
    t = t + eri_warp(A, po[r], s, p, po[q]) * (2.0 * c) - eri_warp(A, s, po[r], p, po[q]) * (2.0 * c);
  }
  {
    const double c = A.l1[p * n + s] + A.l2[p * n + po[s]];
    t = t + eri_warp(A, po[p], q, r, po[s]) * (2.0 * c) - eri_warp(A, po[p], q, po[s], r) * (2.0 * c);
  }
  if (p == po[r]) {
    Cx sum = cx(0.0);
    for (int64_t w = 0; w < n; ++w) sum = sum + eri_warp(A, s, q, w, po[w]) * (A.l1[r * n + w] + A.l2[r * n + po[w]]);
    t = t + sum * 2.0;
  }
  return t;
}

__global__ void joint_diag_kernel(const JointArgs A) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  const int64_t n = A.n;
  for (int64_t I = warp; I < A.npairs; I += nw) {
    const int64_t p = A.pairs[2 * I], q = A.pairs[2 * I + 1];
    auto h2 = [&](int64_t i, int64_t j) { return A.h2[i * n + j]; };
    auto x2 = [&](int64_t i, int64_t j) { return A.x2[i * n + j]; };
    const double np = A.occ[p], nq = A.occ[q];
    const Cx Fpp = at(A.F, n, p, p), Fqq = at(A.F, n, q, q), Hpp = at(A.H, n, p, p), Hqq = at(A.H, n, q, q);
    // G_pq,pq: no delta terms, both leftover integrals eri(q,q,p,p) = Q(q,p)
    const Cx g1 = at(A.Q, n, q, p) * (x2(p, q) - h2(q, q) + x2(p, q) - x2(p, p)) +
                  at(A.Q, n, q, p) * (h2(p, p) + x2(q, q) - x2(p, q) - x2(p, q));
    // G_pq,qp: ftex(p,p) + conj(ftex(q,q)) - h(p,p) n_q - h(q,q) n_p + M(q,p) + M(p,q)
    //          + J(p,q) (...) + K(p,q) (...)
    const Cx g2 = Fpp + conjc(Fqq) - Hpp * nq - Hqq * np + at(A.M, n, q, p) + at(A.M, n, p, q) +
                  at(A.J, n, p, q) * (x2(q, q) - h2(p, q) + x2(p, p) - x2(q, p)) +
                  at(A.K, n, p, q) * (h2(q, p) + x2(q, p) - x2(p, p) - x2(q, q));
    // G_qp,pq
    const Cx g3 = Fqq + conjc(Fpp) - Hqq * np - Hpp * nq + at(A.M, n, p, q) + at(A.M, n, q, p) +
                  at(A.J, n, q, p) * (x2(p, p) - h2(q, p) + x2(q, q) - x2(p, q)) +
                  at(A.K, n, q, p) * (h2(p, q) + x2(p, q) - x2(q, q) - x2(p, p));
    // G_qp,qp: eri(p,p,q,q) = Q(p,q)
    const Cx g4 = at(A.Q, n, p, q) * (x2(q, p) - h2(p, p) + x2(q, p) - x2(q, q)) +
                  at(A.Q, n, p, q) * (h2(q, q) + x2(p, p) - x2(q, p) - x2(q, p));
    Cx a = g1, b = g2, c = g3, e = g4;
    if (A.po) {
      a = a + raw_l(A, p, q, p, q);
      b = b + raw_l(A, p, q, q, p);
      c = c + raw_l(A, q, p, p, q);
      e = e + raw_l(A, q, p, q, p);
    }
    if (lane == 0) {
      A.out[I] = (a - b - c + e).re;
      A.out[A.npairs + I] = -(a + b + c + e).re;
    }
  }
}

// Q(i, j) = sum_P B(P,i,j)^2 (complex).
__global__ void q_matrix_kernel(const double* B, int64_t naux, int64_t n, double* Q) {
  const int64_t n2 = n * n;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n2;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int64_t P = 0; P < naux; ++P) {
      const double x = B[2 * (P * n2 + e)], y = B[2 * (P * n2 + e) + 1];
      re += x * x - y * y;
      im += 2.0 * x * y;
    }
    Q[2 * e] = re;
    Q[2 * e + 1] = im;
  }
}

// D = K - J (complex), h2c = h2 as complex.
__global__ void kmj_kernel(const double* K, const double* J, const double* h2, double* D, double* h2c, int64_t n2) {
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n2;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    D[2 * e] = K[2 * e] - J[2 * e];
    D[2 * e + 1] = K[2 * e + 1] - J[2 * e + 1];
    h2c[2 * e] = h2[e];
    h2c[2 * e + 1] = 0.0;
  }
}

}  // namespace

void mo_hx_joint_hessian_diagonal(rr_mo_store* m, const double* h, const double* occ, const double* h2,
                                  const double* x2, const double* fock, int64_t npairs, const int64_t* pairs,
                                  const int64_t* pair_of, const double* l1, const double* l2, double* out, bool host,
                                  cudaStream_t s) {
  RR_REQUIRE(m->cplx, RR_ERR_UNSUPPORTED,
             "hartreeExchangeJointHessianDiagonal: needs a complex MO tensor (RiMoEri); the reference has no real "
             "joint form");
  const int64_t n = m->n, n2 = n * n;
  std::vector<int64_t> hp(static_cast<size_t>(2 * npairs)), hpo;
  if (npairs > 0)
    RR_CUDA(cudaMemcpy(hp.data(), pairs, sizeof(int64_t) * 2 * npairs, host ? cudaMemcpyHostToHost : cudaMemcpyDeviceToHost));
  for (int64_t i = 0; i < 2 * npairs; i += 2)
    RR_REQUIRE(hp[i] >= 0 && hp[i] < n && hp[i + 1] >= 0 && hp[i + 1] < n && hp[i] != hp[i + 1], RR_ERR_ARG,
               "hartreeExchangeJointHessianDiagonal: pair index out of range or p == q");
  if (pair_of) {
    hpo.resize(static_cast<size_t>(n));
    RR_CUDA(cudaMemcpy(hpo.data(), pair_of, sizeof(int64_t) * n, host ? cudaMemcpyHostToHost : cudaMemcpyDeviceToHost));
    for (int64_t v : hpo) RR_REQUIRE(v >= 0 && v < n, RR_ERR_ARG, "hartreeExchangeJointHessianDiagonal: pair_of out of range");
  }
  Arena ar(&m->io);
  double *Hd, *Fd, *od, *h2d, *x2d, *J, *K, *Q, *M, *D, *h2c, *pd, *pod = nullptr, *l1d = nullptr, *l2d = nullptr, *outd;
  ar.request(&Hd, 2 * n2);
  ar.request(&Fd, 2 * n2);
  ar.request(&od, n);
  ar.request(&h2d, n2);
  ar.request(&x2d, n2);
  ar.request(&J, 2 * n2);
  ar.request(&K, 2 * n2);
  ar.request(&Q, 2 * n2);
  ar.request(&M, 2 * n2);
  ar.request(&D, 2 * n2);
  ar.request(&h2c, 2 * n2);
  ar.request(&pd, 2 * std::max<int64_t>(npairs, 1));
  ar.request(&outd, 2 * std::max<int64_t>(npairs, 1));
  if (pair_of) {
    ar.request(&pod, n);
    ar.request(&l1d, n2);
    ar.request(&l2d, n2);
  }
  ar.commit();
  copy_in(Hd, h, 2 * n2, host, s);
  copy_in(Fd, fock, 2 * n2, host, s);
  copy_in(od, occ, n, host, s);
  copy_in(h2d, h2, n2, host, s);
  copy_in(x2d, x2, n2, host, s);
  if (npairs > 0) RR_CUDA(cudaMemcpyAsync(pd, hp.data(), sizeof(int64_t) * 2 * npairs, cudaMemcpyHostToDevice, s));
  if (pair_of) {
    RR_CUDA(cudaMemcpyAsync(pod, hpo.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice, s));
    copy_in(l1d, l1, n2, host, s);
    copy_in(l2d, l2, n2, host, s);
  }
  mo_jkl(m, nullptr, J, K, nullptr, false, s);
  q_matrix_kernel<<<blocks_for(n2), 256, 0, s>>>(m->B.p, m->naux, n, Q);
  RR_LAUNCH_CHECK();
  kmj_kernel<<<blocks_for(n2), 256, 0, s>>>(K, J, h2d, D, h2c, n2);
  RR_LAUNCH_CHECK();
  GemmDesc g;  // M = two_rdm_h (K - J)
  g.cplx = true;
  g.M = n; g.N = n; g.K = n; g.A = h2c; g.lda = n; g.B = D; g.ldb = n; g.C = M; g.ldc = n;
  gemm(g, s);
  JointArgs A{Hd, Fd, od, h2d, x2d, J, K, Q, M, m->B.p, reinterpret_cast<const int64_t*>(pd),
              pair_of ? reinterpret_cast<const int64_t*>(pod) : nullptr, l1d, l2d, n, m->naux, npairs, outd};
  if (npairs > 0) {
    const int64_t warps = std::min<int64_t>(npairs, 148LL * 64);
    joint_diag_kernel<<<static_cast<int>((warps * 32 + 255) / 256), 256, 0, s>>>(A);
    RR_LAUNCH_CHECK();
  }
  copy_out(out, outd, 2 * npairs, host, s);
}

}  // namespace rr
