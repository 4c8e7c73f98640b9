// The CASSCF RI operators on a resident MO tensor (src/MCSCF/CasFock.cpp:246-262 and the RI primitives
// they call, :74-147): the two-electron operator G(rho) = J(rho) - K(rho) of a one-particle density, the
// active cumulant Fock contraction and the active-space integrals.  For a RiNonRelSpinMoEri the
// reference works on embeddedB() (the 2n spin-orbital tensor); so do these.  No conjugation of B
// anywhere (the reference's GEMMs are plain transposes); K uses the low-rank factors of rho
// (|w| > 1e-14), K = sum_P B_P conj(U) diag(w) U^T B_P.
#include <algorithm>
#include <cmath>
#include <vector>

#include "mo_store.cuh"

namespace rr {
namespace {

int blocks_for(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4736))); }

// ucj (d x nk) = conj(U)(:, keep), uwt (nk x d) = w_keep U(:, keep)^T from the solver's rows
// (row k of R holds eigenvector k, conjugated for the complex solver: U(i, k) = conj(R[k][i])).
template <int PL>
__global__ void low_rank_factors_kernel(const double* R, const double* w, const int* keep, int64_t d, int64_t nk,
                                        double* ucj, double* uwt) {
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < d * nk;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = e / nk, j = e % nk, k = keep[j];
    const double re = R[PL * (k * d + i)], im = PL == 2 ? R[2 * (k * d + i) + 1] : 0.0;  // conj(U(i, k))
    ucj[PL * (i * nk + j)] = re;
    if (PL == 2) ucj[2 * (i * nk + j) + 1] = im;
    const double wk = w[k];
    uwt[PL * (j * d + i)] = wk * re;
    if (PL == 2) uwt[2 * (j * d + i) + 1] = -wk * im;
  }
}

// Bact[P][s a + t] = B[P][act[s] d + act[t]]  (PL planes)
template <int PL>
__global__ void gather_active_kernel(double* Bact, const double* B, const int64_t* act, int64_t naux, int64_t d,
                                     int64_t a) {
  const int64_t a2 = a * a;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < naux * a2;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t P = e / a2, st = e % a2;
    const int64_t src = P * d * d + act[st / a] * d + act[st % a];
    Bact[PL * e] = B[PL * src];
    if (PL == 2) Bact[2 * e + 1] = B[2 * src + 1];
  }
}

// Bsel[(P a + r) d + p] = B[P][act[r] d + p]
template <int PL>
__global__ void gather_rows_kernel(double* Bsel, const double* B, const int64_t* act, int64_t naux, int64_t d,
                                   int64_t a) {
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < naux * a * d;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t Pr = e / d, p = e % d, P = Pr / a, r = Pr % a;
    const int64_t src = P * d * d + act[r] * d + p;
    Bsel[PL * e] = B[PL * src];
    if (PL == 2) Bsel[2 * e + 1] = B[2 * src + 1];
  }
}

// G = jv - K (count doubles)
__global__ void sub_kernel(double* G, const double* jv, const double* K, int64_t count) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    G[i] = jv[i] - K[i];
}

std::vector<int64_t> checked_active(const int64_t* active, int64_t a, int64_t d, bool host) {
  std::vector<int64_t> act(static_cast<size_t>(a));
  if (a > 0)
    RR_CUDA(cudaMemcpy(act.data(), active, sizeof(int64_t) * a, host ? cudaMemcpyHostToHost : cudaMemcpyDeviceToHost));
  for (int64_t v : act) RR_REQUIRE(v >= 0 && v < d, RR_ERR_ARG, "casActiveCumulantFock: active index out of range");
  return act;
}

}  // namespace

void cas_two_electron(rr_mo_store* m, const double* rho, double* G, bool host, cudaStream_t s) {
  const int PL = m->cplx ? 2 : 1;
  int64_t d = 0;
  const double* Bt = mo_operand(m, s, &d);
  const int64_t naux = m->naux, dd = d * d;
  Arena ar(&m->io);
  double *rd, *R, *w, *c, *jv, *Km, *Gd;
  ar.request(&rd, PL * dd);
  ar.request(&R, PL * dd);
  ar.request(&w, d);
  ar.request(&c, PL * std::max<int64_t>(naux, 1));
  ar.request(&jv, PL * dd);
  ar.request(&Km, PL * dd);
  ar.request(&Gd, PL * dd);
  ar.commit();
  copy_in(rd, rho, PL * dd, host, s);
  // Coulomb: c_P = sum_st rho_st B(P, s d + t), J = B^T c   (CasFock.cpp:76-82)
  GemmDesc g1;
  g1.cplx = m->cplx != 0;
  g1.M = naux; g1.N = 1; g1.K = dd; g1.A = Bt; g1.lda = dd; g1.B = rd; g1.ldb = 1; g1.C = c; g1.ldc = 1;
  gemm(g1, s);
  GemmDesc g2;
  g2.cplx = m->cplx != 0;
  g2.M = dd; g2.N = 1; g2.K = naux; g2.A = Bt; g2.lda = dd; g2.opA = Op::T; g2.B = c; g2.ldb = 1; g2.C = jv; g2.ldc = 1;
  if (naux > 0) gemm(g2, s);
  else RR_CUDA(cudaMemsetAsync(jv, 0, sizeof(double) * PL * dd, s));
  // Exchange from the low-rank factors of rho (CasFock.cpp:84-108)
  RR_CUDA(cudaMemcpyAsync(R, rd, sizeof(double) * PL * dd, cudaMemcpyDeviceToDevice, s));
  if (m->cplx) eigh_herm_ctx(m->ctx, R, d, w, s);
  else eigh_sym_ctx(m->ctx, R, d, w, s);
  std::vector<double> wh(static_cast<size_t>(d));
  int info = 0;
  RR_CUDA(cudaMemcpyAsync(wh.data(), w, sizeof(double) * d, cudaMemcpyDeviceToHost, s));
  RR_CUDA(cudaMemcpyAsync(&info, m->ctx.solver_info.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  RR_CUDA(cudaStreamSynchronize(s));
  RR_REQUIRE(info == 0, RR_ERR_SOLVER, "casTwoElectronOperator: the eigensolver of rho did not converge");
  std::vector<int> keep;
  for (int64_t k = 0; k < d; ++k)
    if (std::abs(wh[k]) > 1e-14) keep.push_back(static_cast<int>(k));
  const int64_t nk = static_cast<int64_t>(keep.size());
  RR_CUDA(cudaMemsetAsync(Km, 0, sizeof(double) * PL * dd, s));
  if (nk > 0 && naux > 0) {
    const int64_t per = d * nk;  // doubles of one aux row of each factor product (per plane)
    const int64_t pc = std::max<int64_t>(1, std::min<int64_t>(naux, (16LL << 20) / std::max<int64_t>(per, 1)));
    DevBuf<double> fac(static_cast<size_t>(2 * PL * per + 32)), Aall(static_cast<size_t>(PL * pc * per)),
        Call(static_cast<size_t>(PL * pc * per));
    DevBuf<int> kd(static_cast<size_t>(nk));
    RR_CUDA(cudaMemcpyAsync(kd.p, keep.data(), sizeof(int) * nk, cudaMemcpyHostToDevice, s));
    double* ucj = fac.p;
    double* uwt = fac.p + PL * per;
    if (m->cplx) low_rank_factors_kernel<2><<<blocks_for(d * nk), 256, 0, s>>>(R, w, kd.p, d, nk, ucj, uwt);
    else low_rank_factors_kernel<1><<<blocks_for(d * nk), 256, 0, s>>>(R, w, kd.p, d, nk, ucj, uwt);
    RR_LAUNCH_CHECK();
    for (int64_t P0 = 0; P0 < naux; P0 += pc) {
      const int64_t cnt = std::min(pc, naux - P0);
      GemmDesc a;  // A_P = B_P conj(U)  -> Aall (d x cnt nk), column block P
      a.cplx = m->cplx != 0;
      a.M = d; a.N = nk; a.K = d;
      a.A = Bt + PL * P0 * dd; a.lda = d; a.strideA = dd;
      a.B = ucj; a.ldb = nk; a.strideB = 0;
      a.C = Aall.p; a.ldc = cnt * nk; a.strideC = nk;
      a.batch = cnt;
      gemm(a, s);
      GemmDesc b;  // C_P = diag(w) U^T B_P  -> Call (cnt nk x d), row block P
      b.cplx = m->cplx != 0;
      b.M = nk; b.N = d; b.K = d;
      b.A = uwt; b.lda = d; b.strideA = 0;
      b.B = Bt + PL * P0 * dd; b.ldb = d; b.strideB = dd;
      b.C = Call.p; b.ldc = d; b.strideC = nk * d;
      b.batch = cnt;
      gemm(b, s);
      GemmDesc k;  // K += Aall Call
      k.cplx = m->cplx != 0;
      k.M = d; k.N = d; k.K = cnt * nk;
      k.A = Aall.p; k.lda = cnt * nk; k.B = Call.p; k.ldb = d; k.C = Km; k.ldc = d; k.beta = 1.0;
      m->work.ensure(static_cast<size_t>(std::max<int64_t>(gemm_work_doubles(k), 1)));
      gemm(k, s, m->work.p, static_cast<int64_t>(m->work.n));
    }
    RR_CUDA(cudaStreamSynchronize(s));  // the factor buffers are released at the end of this scope
  }
  sub_kernel<<<blocks_for(PL * dd), 256, 0, s>>>(Gd, jv, Km, PL * dd);
  RR_LAUNCH_CHECK();
  copy_out(G, Gd, PL * dd, host, s);
}

void cas_cumulant_fock(rr_mo_store* m, int64_t a, const int64_t* active, const double* lambda, double* F, bool host,
                       cudaStream_t s) {
  const int PL = m->cplx ? 2 : 1;
  int64_t d = 0;
  const double* Bt = mo_operand(m, s, &d);
  const int64_t naux = m->naux, a2 = a * a;
  const std::vector<int64_t> act = checked_active(active, a, d, host);
  Arena ar(&m->io);
  double *ad, *lam, *Bact, *T, *Bsel, *Fd;
  ar.request(&ad, std::max<int64_t>(a, 1));
  ar.request(&lam, PL * a2 * a2);
  ar.request(&Bact, PL * naux * a2);
  ar.request(&T, PL * naux * a2);
  ar.request(&Bsel, PL * naux * a * d);
  ar.request(&Fd, PL * d * a);
  ar.commit();
  int64_t* actd = reinterpret_cast<int64_t*>(ad);
  if (a > 0) RR_CUDA(cudaMemcpyAsync(actd, act.data(), sizeof(int64_t) * a, cudaMemcpyHostToDevice, s));
  copy_in(lam, lambda, PL * a2 * a2, host, s);
  if (a == 0 || naux == 0) {
    RR_CUDA(cudaMemsetAsync(Fd, 0, sizeof(double) * PL * d * std::max<int64_t>(a, 1), s));
  } else {
    if (m->cplx) gather_active_kernel<2><<<blocks_for(naux * a2), 256, 0, s>>>(Bact, Bt, actd, naux, d, a);
    else gather_active_kernel<1><<<blocks_for(naux * a2), 256, 0, s>>>(Bact, Bt, actd, naux, d, a);
    RR_LAUNCH_CHECK();
    GemmDesc t;  // T = Bact Lambda
    t.cplx = m->cplx != 0;
    t.M = naux; t.N = a2; t.K = a2; t.A = Bact; t.lda = a2; t.B = lam; t.ldb = a2; t.C = T; t.ldc = a2;
    gemm(t, s);
    if (m->cplx) gather_rows_kernel<2><<<blocks_for(naux * a * d), 256, 0, s>>>(Bsel, Bt, actd, naux, d, a);
    else gather_rows_kernel<1><<<blocks_for(naux * a * d), 256, 0, s>>>(Bsel, Bt, actd, naux, d, a);
    RR_LAUNCH_CHECK();
    GemmDesc f;  // F = Bsel^T T over the (P, r) rows
    f.cplx = m->cplx != 0;
    f.M = d; f.N = a; f.K = naux * a; f.A = Bsel; f.lda = d; f.opA = Op::T; f.B = T; f.ldb = a; f.C = Fd; f.ldc = a;
    m->work.ensure(static_cast<size_t>(std::max<int64_t>(gemm_work_doubles(f), 1)));
    gemm(f, s, m->work.p, static_cast<int64_t>(m->work.n));
  }
  copy_out(F, Fd, PL * d * a, host, s);
}

void cas_active_integrals(rr_mo_store* m, int64_t a, const int64_t* active, double* out, bool host, cudaStream_t s) {
  const int PL = m->cplx ? 2 : 1;
  int64_t d = 0;
  const double* Bt = mo_operand(m, s, &d);
  const int64_t naux = m->naux, a2 = a * a;
  const std::vector<int64_t> act = checked_active(active, a, d, host);
  Arena ar(&m->io);
  double *ad, *Bact, *O;
  ar.request(&ad, std::max<int64_t>(a, 1));
  ar.request(&Bact, PL * naux * a2);
  ar.request(&O, PL * a2 * a2);
  ar.commit();
  int64_t* actd = reinterpret_cast<int64_t*>(ad);
  if (a == 0) return;
  RR_CUDA(cudaMemcpyAsync(actd, act.data(), sizeof(int64_t) * a, cudaMemcpyHostToDevice, s));
  if (naux == 0) {
    RR_CUDA(cudaMemsetAsync(O, 0, sizeof(double) * PL * a2 * a2, s));
  } else {
    if (m->cplx) gather_active_kernel<2><<<blocks_for(naux * a2), 256, 0, s>>>(Bact, Bt, actd, naux, d, a);
    else gather_active_kernel<1><<<blocks_for(naux * a2), 256, 0, s>>>(Bact, Bt, actd, naux, d, a);
    RR_LAUNCH_CHECK();
    GemmDesc g;  // (tu|vw) = sum_P Bact(P, tu) Bact(P, vw)
    g.cplx = m->cplx != 0;
    g.M = a2; g.N = a2; g.K = naux; g.A = Bact; g.lda = a2; g.opA = Op::T; g.B = Bact; g.ldb = a2; g.C = O; g.ldc = a2;
    m->work.ensure(static_cast<size_t>(std::max<int64_t>(gemm_work_doubles(g), 1)));
    gemm(g, s, m->work.p, static_cast<int64_t>(m->work.n));
  }
  copy_out(out, O, PL * a2 * a2, host, s);
}

}  // namespace rr
