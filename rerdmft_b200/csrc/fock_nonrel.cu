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
void coulomb_pass2_release(rr_ri_store* h, cudaStream_t s);

// release_pass2: right after the half-transform, release the pending J pass 2 onto the side stream
// so that it overlaps the compute-bound SYRK.
void exchange_nonrel(rr_ri_store* h, const double* Ct, int64_t ldct, bool ct_transposed, int64_t nocc, double* K,
                     cudaStream_t s, bool release_pass2 = false) {
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
  if (release_pass2) coulomb_pass2_release(h, s);

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
  JPlan pl = j_plan(1, &t, h->naux, 1);
  h->jscr.ensure(static_cast<size_t>(round_up(pl.gpart_doubles, 32) + pl.jpart_doubles + 32));
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

// Same for one or two tensors sharing gamma (4c: LL and SS); Dp[t] pitched, J[t] dense outputs.
void coulomb_async_multi(rr_ri_store* h, int ntens, const double* const* Dp, double* const* J, cudaStream_t s) {
  JTensor t[2];
  const int64_t nn[2] = {h->n, h->ns};
  for (int i = 0; i < ntens; ++i) {
    t[i].B = h->B[i].p;
    t[i].pitch = h->pitch[i];
    t[i].len = nn[i] * nn[i];
    t[i].D = Dp[i];
    t[i].J = J[i];
  }
  JPlan pl = j_plan(ntens, t, h->naux, 1);
  h->jscr.ensure(static_cast<size_t>(round_up(pl.gpart_doubles, 32) + pl.jpart_doubles + 32));
  double* gpart = h->jscr.p;
  double* jpart = h->jscr.p + round_up(pl.gpart_doubles, 32);
  auto& c = h->ctx;
  RR_CUDA(cudaEventRecord(c.fork, s));
  RR_CUDA(cudaStreamWaitEvent(c.side, c.fork, 0));
  prof_mark(h, 5, c.side);
  j_pass1(pl, gpart, h->status.p, c.side);
  j_pass2(pl, gpart, jpart, h->status.p, c.side);
  j_finish(pl, jpart, 1.0, c.side);
  prof_mark(h, 6, c.side);
  RR_CUDA(cudaEventRecord(c.join, c.side));
}

// Two-phase J for the nonrelativistic build: pass 1 starts on the side stream at once (it only
// needs D and overlaps the occupied recovery); pass 2 waits for the `mid` event, recorded on the
// main stream after the half-transform, so it overlaps the compute-bound SYRK instead of competing
// with the half-transform for HBM.
void coulomb_split_async(rr_ri_store* h, const double* Dp, double* J, cudaStream_t s) {
  JTensor t;
  t.B = h->B[0].p;
  t.pitch = h->pitch[0];
  t.len = h->n * h->n;
  t.D = Dp;
  t.J = J;
  JPlan pl = j_plan(1, &t, h->naux, 1);
  h->jscr.ensure(static_cast<size_t>(round_up(pl.gpart_doubles, 32) + pl.jpart_doubles + 32));
  double* gpart = h->jscr.p;
  double* jpart = h->jscr.p + round_up(pl.gpart_doubles, 32);
  auto& c = h->ctx;
  if (!c.mid) RR_CUDA(cudaEventCreateWithFlags(&c.mid, cudaEventDisableTiming));
  RR_CUDA(cudaEventRecord(c.fork, s));
  RR_CUDA(cudaStreamWaitEvent(c.side, c.fork, 0));
  prof_mark(h, 5, c.side);
  j_pass1(pl, gpart, h->status.p, c.side);
  h->pending_pass2 = pl;
  h->pending_gpart = gpart;
  h->pending_jpart = jpart;
  h->has_pending_pass2 = true;
}

void coulomb_pass2_release(rr_ri_store* h, cudaStream_t s) {
  if (!h->has_pending_pass2) return;
  auto& c = h->ctx;
  RR_CUDA(cudaEventRecord(c.mid, s));
  RR_CUDA(cudaStreamWaitEvent(c.side, c.mid, 0));
  j_pass2(h->pending_pass2, h->pending_gpart, h->pending_jpart, h->status.p, c.side);
  j_finish(h->pending_pass2, h->pending_jpart, 1.0, c.side);
  prof_mark(h, 6, c.side);
  RR_CUDA(cudaEventRecord(c.join, c.side));
  h->has_pending_pass2 = false;
}

void coulomb_join(rr_ri_store* h, cudaStream_t s) { RR_CUDA(cudaStreamWaitEvent(s, h->ctx.join, 0)); }

int64_t occupied_ct(rr_ri_store* h, const double* X, const double* S, const double* Dp, int64_t n, int64_t n_eff,
                    double scale, bool cplx, bool weighted, double* Ct, cudaStream_t s);

void fock_nonrel(rr_ri_store* h, const double* hc, const double* D, const double* S, const double* X, int64_t n_eff,
                 double* F, const rr_opts* o) {
  RR_REQUIRE(h->ntens == 1, RR_ERR_STATE, "rr_ri_fock_nonrel: handle holds a 4-component store");
  const int64_t n = h->n, n2 = n * n;
  RR_REQUIRE(n_eff >= 0 && n_eff <= n, RR_ERR_ARG, "rr_ri_fock_nonrel: n_eff out of range");
  const bool host = !o || o->mem == RR_MEM_HOST;
  cudaStream_t s = call_stream(h, o);
  const int64_t pitch = round_up(std::max<int64_t>(n2, 2), 32);

  double *Dp, *hd, *Sd, *Xd, *Fd, *J, *K, *Ct;
  Arena ar(&h->mats);
  ar.request(&Dp, pitch);
  ar.request(&J, n2);
  ar.request(&K, n2);
  ar.request(&Ct, n * std::max<int64_t>(n_eff, 1));
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
  // J pass 1 on the side stream alongside the occupied recovery (X^T (S D S / 2) X, eigenvalues
  // > 0.5, as c_t = F^T X^T); J pass 2 alongside the SYRK.
  coulomb_split_async(h, Dp, J, s);
  const int64_t nocc = occupied_ct(h, Xd, Sd, Dp, n, n_eff, 0.5, false, false, Ct, s);
  prof_mark(h, 1, s);
  exchange_nonrel(h, Ct, n, false, nocc, K, s, true);
  coulomb_pass2_release(h, s);  // no-op unless the exchange had nothing to transform
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
  coulomb_split_async(h, Dp, J, s);
  prof_mark(h, 1, s);
  exchange_nonrel(h, Cd, nocc, true, nocc, K, s, true);
  coulomb_pass2_release(h, s);
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
