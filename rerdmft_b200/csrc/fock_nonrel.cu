// Nonrelativistic RI Fock build (reference: src/NON_REL/NonRelFockMatrixRi.cpp:71-143).
//
// Schedule for one call (stream `s` plus the handle's side stream):
//   side: J pass 1 (gamma = B vec D) -> J pass 2 (J = B^T gamma) -> J finish     [HBM-bound]
//   main: occupied recovery (S D S, X^T (.) X / 2, dsyevd, C_occ^T = Y_occ^T X^T)
//         half-transform T[P] = C_occ^T B^P (batched DMMA GEMM)                  [FP64 tensor]
//         K' = sum_P T[P]^T T[P] (split-K DMMA SYRK, upper tiles + mirror)        [FP64 tensor]
//   join, F = h + J - K'   (K' = K/2 of the reference: its c_t carries sqrt(2)).
#include <algorithm>

#include "ri_store.cuh"

namespace rr {

namespace {

// D = 2 C C^T  (C: n x nocc row-major) into a pitched buffer.
void density_from_occupied(double* Dp, const double* C, int64_t n, int64_t nocc, cudaStream_t s, double* work,
                           int64_t work_cap) {
  GemmDesc g;
  g.M = n; g.N = n; g.K = nocc;
  g.A = C; g.lda = nocc; g.opA = Op::N;
  g.B = C; g.ldb = nocc; g.opB = Op::T;
  g.C = Dp; g.ldc = n;
  g.alpha = 2.0;
  gemm(g, s, work, work_cap);
}

}  // namespace

// Exchange K' = sum_P (Ct B^P)^T (Ct B^P) for a given Ct (nocc x n, row-major with leading
// dimension ldct, or its transpose when ct_transposed: Ct = C^T with C stored n x nocc).
void exchange_nonrel(rr_ri_store* h, const double* Ct, int64_t ldct, bool ct_transposed, int64_t nocc, double* K,
                     cudaStream_t s) {
  const int64_t n = h->n, naux = h->naux;
  if (nocc == 0 || naux == 0) {
    RR_CUDA(cudaMemsetAsync(K, 0, sizeof(double) * n * n, s));
    return;
  }
  h->T.ensure(static_cast<size_t>(naux * nocc * n));
  GemmDesc ht;
  ht.M = nocc; ht.N = n; ht.K = n;
  ht.A = Ct; ht.lda = ldct; ht.opA = ct_transposed ? Op::T : Op::N; ht.strideA = 0;
  ht.B = h->B[0].p; ht.ldb = n; ht.opB = Op::N; ht.strideB = h->pitch[0];
  ht.C = h->T.p; ht.ldc = n; ht.strideC = nocc * n;
  ht.batch = naux;
  gemm(ht, s);
  prof_mark(h, 2, s);

  GemmDesc sk;
  sk.M = n; sk.N = n; sk.K = naux * nocc;
  sk.A = h->T.p; sk.lda = n; sk.opA = Op::T;
  sk.B = h->T.p; sk.ldb = n; sk.opB = Op::N;
  sk.C = K; sk.ldc = n;
  sk.mirror = 1;
  const int64_t want = gemm_work_doubles(sk);
  h->work.ensure(static_cast<size_t>(std::max<int64_t>(want, 1)));
  gemm(sk, s, h->work.p, static_cast<int64_t>(h->work.n));
}

// Launches the J passes for the pitched density Dp on the side stream, forked from / joined to s.
void coulomb_async(rr_ri_store* h, const double* Dp, double* J, double scale, cudaStream_t s) {
  JTensor t;
  t.B = h->B[0].p;
  t.pitch = h->pitch[0];
  t.len = h->n * h->n;
  t.D = Dp;
  t.J = J;
  JPlan pl = j_plan(1, &t, h->naux);
  h->jscr.ensure(static_cast<size_t>(pl.gpart_doubles + pl.jpart_doubles + 32));
  double* gpart = h->jscr.p;
  double* jpart = h->jscr.p + round_up(pl.gpart_doubles, 32);
  auto& c = h->ctx;
  RR_CUDA(cudaEventRecord(c.fork, s));
  RR_CUDA(cudaStreamWaitEvent(c.side, c.fork, 0));
  prof_mark(h, 5, c.side);
  j_pass1(pl, gpart, h->status.p, c.side);
  j_pass2(pl, gpart, jpart, h->status.p, c.side);
  j_finish(pl, jpart, scale, c.side);
  prof_mark(h, 6, c.side);
  RR_CUDA(cudaEventRecord(c.join, c.side));
}

void coulomb_join(rr_ri_store* h, cudaStream_t s) { RR_CUDA(cudaStreamWaitEvent(s, h->ctx.join, 0)); }

void fock_nonrel(rr_ri_store* h, const double* hc, const double* D, const double* S, const double* X, int64_t n_eff,
                 double* F, const rr_opts* o) {
  RR_REQUIRE(h->ntens == 1, RR_ERR_STATE, "rr_ri_fock_nonrel: handle holds a 4-component store");
  const int64_t n = h->n, n2 = n * n;
  RR_REQUIRE(n_eff >= 0 && n_eff <= n, RR_ERR_ARG, "rr_ri_fock_nonrel: n_eff out of range");
  const bool host = !o || o->mem == RR_MEM_HOST;
  cudaStream_t s = call_stream(h, o);
  const int64_t pitch = round_up(std::max<int64_t>(n2, 2), 32);

  double *Dp, *hd, *Sd, *Xd, *Fd, *J, *K, *SD, *SDS, *Y, *Pe, *W, *Ct;
  Arena ar(&h->mats);
  ar.request(&Dp, pitch);
  ar.request(&J, n2);
  ar.request(&K, n2);
  ar.request(&SD, n2);
  ar.request(&SDS, n2);
  ar.request(&Y, n * n_eff);
  ar.request(&Pe, n_eff * n_eff);
  ar.request(&W, n_eff);
  ar.request(&Ct, n * n_eff);
  if (host) {
    ar.request(&hd, n2);
    ar.request(&Sd, n2);
    ar.request(&Xd, n * n_eff);
    ar.request(&Fd, n2);
  }
  ar.commit();
  if (!host) { hd = const_cast<double*>(hc); Sd = const_cast<double*>(S); Xd = const_cast<double*>(X); Fd = F; }

  prof_mark(h, 0, s);
  copy_in_padded(Dp, pitch, D, n2, host, s);
  if (host) {
    copy_in(hd, hc, n2, true, s);
    copy_in(Sd, S, n2, true, s);
    copy_in(Xd, X, n * n_eff, true, s);
  }
  coulomb_async(h, Dp, J, 1.0, s);

  // Occupied recovery: P_eff = X^T (S D S / 2) X, keep eigenvalues > 0.5.
  GemmDesc g;
  g.M = n; g.N = n; g.K = n;
  g.A = Sd; g.lda = n; g.B = Dp; g.ldb = n; g.C = SD; g.ldc = n;
  gemm(g, s);
  g.A = SD; g.B = Sd; g.C = SDS;
  gemm(g, s);
  g.N = n_eff; g.A = SDS; g.B = Xd; g.ldb = n_eff; g.C = Y; g.ldc = n_eff;
  gemm(g, s);
  GemmDesc pe;
  pe.M = n_eff; pe.N = n_eff; pe.K = n;
  pe.A = Xd; pe.lda = n_eff; pe.opA = Op::T;
  pe.B = Y; pe.ldb = n_eff; pe.C = Pe; pe.ldc = n_eff; pe.alpha = 0.5;
  gemm(pe, s);
  eigh_sym(h, Pe, n_eff, W, s);
  h->host_w.resize(static_cast<size_t>(std::max<int64_t>(n_eff, 1)));
  if (n_eff) RR_CUDA(cudaMemcpyAsync(h->host_w.data(), W, sizeof(double) * n_eff, cudaMemcpyDeviceToHost, s));
  RR_CUDA(cudaStreamSynchronize(s));
  int info = 0;
  if (n_eff) {
    RR_CUDA(cudaMemcpy(&info, h->ctx.solver_info.p, sizeof(int), cudaMemcpyDeviceToHost));
    RR_REQUIRE(info == 0, RR_ERR_SOLVER, "rr_ri_fock_nonrel: dsyevd failed to converge");
  }
  int64_t nocc = 0;
  for (int64_t i = 0; i < n_eff; ++i) nocc += h->host_w[static_cast<size_t>(i)] > 0.5 ? 1 : 0;
  // Eigenvalues ascend, so the kept eigenvectors are the last nocc rows of Pe (row j = vector j).
  if (nocc) {
    GemmDesc ct;
    ct.M = nocc; ct.N = n; ct.K = n_eff;
    ct.A = Pe + (n_eff - nocc) * n_eff; ct.lda = n_eff;
    ct.B = Xd; ct.ldb = n_eff; ct.opB = Op::T;
    ct.C = Ct; ct.ldc = n;
    gemm(ct, s);
  }
  prof_mark(h, 1, s);
  exchange_nonrel(h, Ct, n, false, nocc, K, s);
  prof_mark(h, 3, s);
  coulomb_join(h, s);
  fock_combine(Fd, hd, J, K, n2, s);
  if (host) copy_out(F, Fd, n2, true, s);
  prof_mark(h, 4, s);
  if (host || (o && o->sync)) check_status(h, s);
}

void jk_occupied(rr_ri_store* h, const double* C, int64_t nocc, double* Jout, double* Kout, const rr_opts* o) {
  RR_REQUIRE(h->ntens == 1, RR_ERR_STATE, "rr_ri_jk_occupied: handle holds a 4-component store");
  RR_REQUIRE(nocc >= 0 && nocc <= h->n, RR_ERR_ARG, "rr_ri_jk_occupied: n_occ out of range");
  const int64_t n = h->n, n2 = n * n;
  const bool host = !o || o->mem == RR_MEM_HOST;
  cudaStream_t s = call_stream(h, o);
  const int64_t pitch = round_up(std::max<int64_t>(n2, 2), 32);
  double *Dp, *Cd, *J, *K;
  Arena ar(&h->mats);
  ar.request(&Dp, pitch);
  if (host) {
    ar.request(&Cd, n * nocc);
    ar.request(&J, n2);
    ar.request(&K, n2);
  }
  ar.commit();
  prof_mark(h, 0, s);
  if (host) copy_in(Cd, C, n * nocc, true, s);
  else { Cd = const_cast<double*>(C); J = Jout; K = Kout; }
  RR_CUDA(cudaMemsetAsync(Dp + n2, 0, sizeof(double) * (pitch - n2), s));
  if (nocc) {
    density_from_occupied(Dp, Cd, n, nocc, s, nullptr, 0);
  } else {
    RR_CUDA(cudaMemsetAsync(Dp, 0, sizeof(double) * n2, s));
  }
  coulomb_async(h, Dp, J, 1.0, s);
  prof_mark(h, 1, s);
  exchange_nonrel(h, Cd, nocc, true, nocc, K, s);
  prof_mark(h, 3, s);
  coulomb_join(h, s);
  if (host) {
    copy_out(Jout, J, n2, true, s);
    copy_out(Kout, K, n2, true, s);
  }
  prof_mark(h, 4, s);
  if (host || (o && o->sync)) check_status(h, s);
}

}  // namespace rr
