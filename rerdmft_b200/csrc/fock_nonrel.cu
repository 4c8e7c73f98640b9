// Nonrelativistic RI Fock build (reference: src/NON_REL/NonRelFockMatrixRi.cpp:71-143).
//
// Schedule for one call (stream `s` plus the handle's side stream):
//   side: J pass 1 (gamma = B vec D) -> J pass 2 (J = B^T gamma) -> J finish     [HBM-bound]
//   main: occupied recovery (S D S, X^T (.) X / 2, dsyevd, C_occ^T = Y_occ^T X^T)
//         half-transform T[P] = C_occ^T B^P (batched DMMA GEMM)                  [FP64 tensor]
//         K' = sum_P T[P]^T T[P] (split-K DMMA SYRK, upper tiles + mirror)        [FP64 tensor]
//   join, F = h + J - K'   (K' = K/2 of the reference: its c_t carries sqrt(2)).
#include <algorithm>
#include <vector>

#include <cstdlib>

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

// The Coulomb passes of the nonrelativistic builds (defined below).
void coulomb_after_ht(rr_ri_store* h, const double* Dp, const double* Ct, int64_t nocc, double* J,
                      const double* tgam, int tseg, cudaStream_t s);
void coulomb_prep(rr_ri_store* h, const double* Dp, const double* Ct, int64_t nocc, double* J, bool have_tgam,
                  cudaStream_t s, bool overlap);
void coulomb_run(rr_ri_store* h, const double* tgam, int tseg, cudaStream_t s);
void coulomb_join(rr_ri_store* h, cudaStream_t s);

namespace {

// K = sum_c parts[c] in the order c = 0, 1, ... (n2 entries each).
__global__ void sum_parts_kernel(double* K, const double* parts, int nparts, int64_t n2) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n2;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double v = parts[i];
    for (int c = 1; c < nparts; ++c) v += parts[c * n2 + i];
    K[i] = v;
  }
}

}  // namespace

// The exchange with the half-transform and the SYRK pipelined over `chunks` ranges of aux indices: the
// main stream half-transforms range c + 1 while the handle's second compute stream runs the SYRK of
// range c into its own partial K_c; K = sum_c K_c in a fixed order.  Needs the m16 half-transform's
// operands (even n and pitch, 16-byte aligned Ct).
void exchange_pipelined(rr_ri_store* h, const double* Ct, int64_t nocc, double* K, cudaStream_t s, int chunks) {
  const int64_t n = h->n, naux = h->naux, n2 = n * n;
  auto& c = h->ctx;
  h->T.ensure(static_cast<size_t>(naux * nocc * n));
  h->kpart.ensure(static_cast<size_t>(chunks * n2));
  std::vector<GemmDesc> sk(chunks);
  std::vector<int64_t> p0(chunks + 1);
  int64_t want = 1;
  for (int ci = 0; ci <= chunks; ++ci) p0[ci] = naux * ci / chunks;
  for (int ci = 0; ci < chunks; ++ci) {
    GemmDesc& g = sk[ci];
    g.M = n; g.N = n; g.K = (p0[ci + 1] - p0[ci]) * nocc;
    g.A = h->T.p + p0[ci] * nocc * n; g.lda = n; g.opA = Op::T;
    g.B = g.A; g.ldb = n; g.opB = Op::N;
    g.C = h->kpart.p + ci * n2; g.ldc = n;
    g.mirror = 1;
    want = std::max(want, gemm_work_doubles(g));
  }
  h->work.ensure(static_cast<size_t>(want));
  for (int ci = 0; ci < chunks; ++ci) {
    RR_REQUIRE(half_transform_m16(Ct, nocc, h->B[0].p + p0[ci] * h->pitch[0], h->pitch[0], p0[ci + 1] - p0[ci], n,
                                  h->T.p + p0[ci] * nocc * n, s, half_transform_config()),
               RR_ERR_STATE, "exchange_pipelined: operands not supported by the m16 half-transform");
    RR_CUDA(cudaEventRecord(c.pipe_ev[ci], s));
    RR_CUDA(cudaStreamWaitEvent(c.pipe_stream, c.pipe_ev[ci], 0));
    gemm(sk[ci], c.pipe_stream, h->work.p, static_cast<int64_t>(h->work.n));
  }
  prof_mark(h, 2, s);
  RR_CUDA(cudaEventRecord(c.pipe_ev[chunks], c.pipe_stream));
  RR_CUDA(cudaStreamWaitEvent(s, c.pipe_ev[chunks], 0));
  sum_parts_kernel<<<static_cast<int>(std::min<int64_t>((n2 + 255) / 256, 1184)), 256, 0, s>>>(K, h->kpart.p, chunks,
                                                                                               n2);
  RR_LAUNCH_CHECK();
}

// Exchange K' = sum_P (Ct B^P)^T (Ct B^P) for a given Ct (nocc x n, row-major with leading
// dimension ldct, or its transpose when ct_transposed: Ct = C^T with C stored n x nocc).
// With Dp given (the SCF loop's FP64 build), the Coulomb matrix J of the pitched density Dp is
// prepared on the side stream beside the half-transform and streamed beside the SYRK
// (coulomb_prep / coulomb_run, gamma from the half-transform epilogue); it lands in Jout; join with
// coulomb_join.  The drop-in build starts its J passes itself (coulomb_early) and passes no Dp.
void exchange_nonrel(rr_ri_store* h, const double* Ct, int64_t ldct, bool ct_transposed, int64_t nocc, double* K,
                     cudaStream_t s, const double* Dp = nullptr, double* Jout = nullptr, bool half_only = false) {
  const int64_t n = h->n, naux = h->naux;
  if (nocc == 0 || naux == 0) {
    if (K) RR_CUDA(cudaMemsetAsync(K, 0, sizeof(double) * n * n, s));
    if (Dp) coulomb_after_ht(h, Dp, Ct, 0, Jout, nullptr, 0, s);
    return;
  }
  h->T.ensure(static_cast<size_t>(naux * nocc * n));
  GemmDesc ht;
  ht.M = nocc; ht.N = n; ht.K = n;
  ht.A = Ct; ht.lda = ldct; ht.opA = ct_transposed ? Op::T : Op::N; ht.strideA = 0;
  ht.B = h->B[0].p; ht.ldb = n; ht.opB = Op::N; ht.strideB = h->pitch[0];
  ht.C = h->T.p; ht.ldc = n; ht.strideC = nocc * n;
  ht.batch = naux;
  // RR_HT_PIPELINE=<chunks> (2 .. 8, for measurement): the drop-in build's half-transform and SYRK
  // pipelined over that many ranges of aux indices (exchange_pipelined).  Both are DMMA-bound, so running
  // them side by side gains nothing and the smaller per-chunk SYRKs cost: at n = 400, naux = 1600,
  // nocc = 40, 1.609 / 1.627 / 1.672 / 1.723 ms per build with 2 / 3 / 4 / 6 chunks against 1.566 ms.
  static const int pipe_chunks = [] {
    const char* e = std::getenv("RR_HT_PIPELINE");
    const int k = e ? std::atoi(e) : 0;
    return k >= 2 && k <= Context::kPipeMax ? k : 0;
  }();
  auto al16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
  if (pipe_chunks && !Dp && !half_only && K && !ct_transposed && ldct == n && half_transform_kind() == 1 &&
      n % 2 == 0 && h->pitch[0] % 2 == 0 && al16(Ct) && naux >= 8 * pipe_chunks) {
    exchange_pipelined(h, Ct, nocc, K, s, pipe_chunks);
    return;
  }
  double* tgam = nullptr;
  int tseg = 0;
  if (Dp) {
    // gamma partials from the half-transform epilogue: 2 * sum T[P] . Ct per output tile
    RR_REQUIRE(!ct_transposed && ldct == n, RR_ERR_STATE, "exchange_nonrel: Coulomb from T needs row-major c_t");
    tseg = static_cast<int>(gemm_tiles_per_batch(ht));
    h->tgam.ensure(static_cast<size_t>(std::max<int64_t>(naux * tseg, 1)));
    tgam = h->tgam.p;
    ht.edot_E = Ct;
    ht.edot_ld = n;
    ht.edot_scale = 2.0;
    ht.edot_out = tgam;
    coulomb_prep(h, Dp, Ct, nocc, Jout, true, s, true);  // side stream, beside the half-transform
  }
  if (!(tgam == nullptr && !ct_transposed && ldct == n && half_transform_kind() == 1 &&
        half_transform_m16(Ct, nocc, h->B[0].p, h->pitch[0], naux, n, h->T.p, s, half_transform_config())))
    gemm(ht, s);
  prof_mark(h, 2, s);
  if (Dp) coulomb_run(h, tgam, tseg, s);  // side stream, beside the SYRK
  if (half_only) return;  // the caller uses T itself (energy-only evaluation)

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

// Energy-only FP64 evaluation of the nonrelativistic build for D = 2 Ct^T Ct (Ct: nocc x n, row-major):
// J from the same passes as the build (J written to Jout) and the half-transform T^P = Ct B^P, then
// energy[0] = 1/2 <D, J> and energy[1] = sum_P ||T^P Ct^T||_F^2 = Tr[D K'] / 2 (F = h + J - K'), so
// 1/2 Tr[D (h + F)] = Tr[D h] + energy[0] - energy[1], without the n x n exchange product.
void energy_nonrel(rr_ri_store* h, const double* Ct, int64_t nocc, const double* Dp, double* Jout, double* energy,
                   cudaStream_t s) {
  const int64_t n = h->n, naux = h->naux;
  exchange_nonrel(h, Ct, n, false, nocc, nullptr, s, Dp, Jout, true);
  h->work.ensure(static_cast<size_t>(std::max<int64_t>(static_cast<int64_t>(h->work.n), naux * nocc * nocc + 256)));
  double* part = h->work.p + naux * nocc * nocc;
  if (nocc > 0 && naux > 0) {
    GemmDesc q;  // Q^P = T^P Ct^T (nocc x nocc)
    q.M = nocc; q.N = nocc; q.K = n;
    q.A = h->T.p; q.lda = n; q.strideA = nocc * n;
    q.B = Ct; q.ldb = n; q.opB = Op::T; q.strideB = 0;
    q.C = h->work.p; q.ldc = nocc; q.strideC = nocc * nocc;
    q.batch = naux;
    gemm(q, s);
    dot_sum(h->work.p, nullptr, naux * nocc * nocc, 1.0, energy + 1, false, part, s);
  } else {
    RR_CUDA(cudaMemsetAsync(energy + 1, 0, sizeof(double), s));
  }
  coulomb_join(h, s);
  dot_sum(Dp, Jout, n * n, 0.5, energy, false, part, s);
}

void pack_for_j(rr_ri_store* h, int t, int64_t n, cudaStream_t s) {
  h->Bpk[t].release();
  h->pitch_pk[t] = 0;
  if (h->naux == 0 || n < 2) return;
  size_t free_b = 0, total_b = 0;
  RR_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const double bytes = 8.0 * static_cast<double>(h->naux) * static_cast<double>(round_up(tri_len(n), 32));
  if (bytes > 0.5 * static_cast<double>(free_b)) return;
  try {
    j_pack_upper(h->B[t].p, h->pitch[t], h->naux, n, h->Bpk[t], h->pitch_pk[t], s);
  } catch (const Error& e) {
    if (e.code != RR_ERR_CUDA) throw;
    // the packed copy is optional: without it J streams B itself (an out-of-memory is not sticky)
    cudaGetLastError();
    h->Bpk[t].release();
    h->pitch_pk[t] = 0;
  }
}

JTensor j_tensor(rr_ri_store* h, int t, int64_t n, const double* D, double* J, int64_t doff, cudaStream_t s) {
  JTensor jt;
  jt.J = J;
  if (h->Bpk[t].p) {
    RR_REQUIRE(static_cast<int64_t>(h->dfold.n) >= doff + tri_len(n) + 1, RR_ERR_ARG, "j_tensor: fold buffer too small");
    j_fold_density(D, n, h->dfold.p + doff, s);
    jt.B = h->Bpk[t].p;
    jt.pitch = h->pitch_pk[t];
    jt.len = tri_len(n);
    jt.tri_n = n;
    jt.D = h->dfold.p + doff;
  } else {
    jt.B = h->B[t].p;
    jt.pitch = h->pitch[t];
    jt.len = n * n;
    jt.D = D;
  }
  return jt;
}

// Same for one or two tensors sharing gamma (4c: LL and SS); Dp[t] pitched, J[t] dense outputs.
void coulomb_async_multi(rr_ri_store* h, int ntens, const double* const* Dp, double* const* J, cudaStream_t s) {
  JTensor t[2];
  const int64_t nn[2] = {h->n, h->ns};
  const int64_t doff1 = round_up(tri_len(nn[0]) + 1, 32);
  h->dfold.ensure(static_cast<size_t>(doff1 + (ntens > 1 ? tri_len(nn[1]) + 1 : 0)));
  for (int i = 0; i < ntens; ++i) t[i] = j_tensor(h, i, nn[i], Dp[i], J[i], i ? doff1 : 0, s);
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

namespace {

__device__ __forceinline__ void atomic_max_pos(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(__double_as_longlong(v)));
}

// m[0] = max |D - Drec|, m[1] = max |D| (m zeroed by the caller).
__global__ void density_diff_kernel(const double* D, const double* Drec, int64_t n2, double* m) {
  __shared__ double r0[32], r1[32];
  double md = 0.0, mx = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n2;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    md = fmax(md, fabs(D[i] - Drec[i]));
    mx = fmax(mx, fabs(D[i]));
  }
  for (int o = 16; o > 0; o >>= 1) {
    md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) { r0[threadIdx.x >> 5] = md; r1[threadIdx.x >> 5] = mx; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) { a = fmax(a, r0[w]); b = fmax(b, r1[w]); }
    atomic_max_pos(m, a);
    atomic_max_pos(m + 1, b);
  }
}

// flag = 1 when the density equals 2 C C^T of the recovered orbitals to 1e-13 relative.
__global__ void density_flag_kernel(const double* m, int* flag) { flag[0] = m[0] <= 1e-13 * fmax(1.0, m[1]) ? 1 : 0; }

}  // namespace

// Coulomb for the nonrelativistic build.  The half-transform GEMM produces, in its epilogue,
// gamma partials from T:  gamma_P = sum_mn B^P_mn D_mn = 2 sum_{i,a} T[P](i,a) Ct(i,a) whenever
// D = 2 Ct^T Ct.  coulomb_prep checks that identity on the device (Drec = 2 Ct^T Ct vs D) and folds D
// onto the packed triangles; coulomb_run (after the half-transform) launches pass 1, which streams B
// only when the check failed (it is launched either way and exits at once when not needed), pass 2
// and the finish.
// Without overlap everything runs on `s` itself and the passes use the whole GPU (3 CTAs per SM).
// With overlap the preparation runs on the side stream beside the half-transform and the passes,
// with one CTA per SM, beside the exchange SYRK that s runs after it: the J kernels are held to 48
// registers so that one of them and two SYRK CTAs (2 x 25.6k registers) fit on an SM together.
// Either way the caller joins with coulomb_join.  have_tgam: the half-transform writes the partials.
void coulomb_prep(rr_ri_store* h, const double* Dp, const double* Ct, int64_t nocc, double* J, bool have_tgam,
                  cudaStream_t s_in, bool overlap) {
  const int64_t n = h->n, naux = h->naux, n2 = n * n;
  auto& c = h->ctx;
  cudaStream_t s = s_in;
  if (overlap) {
    RR_CUDA(cudaEventRecord(c.fork, s_in));
    RR_CUDA(cudaStreamWaitEvent(c.side, c.fork, 0));
    s = c.side;
  }
  h->dfold.ensure(static_cast<size_t>(tri_len(n) + 1));
  JTensor t = j_tensor(h, 0, n, Dp, J, 0, s);
  JPlan pl = j_plan(1, &t, naux, overlap ? 1 : 3);
  const int64_t goff = round_up(pl.gpart_doubles, 32), joff = goff + round_up(pl.jpart_doubles, 32);
  const int64_t toff = joff + round_up(n2, 32);
  h->jscr.ensure(static_cast<size_t>(toff + 64));
  double* Drec = h->jscr.p + joff;
  double* mm = h->jscr.p + toff;
  int* flag = reinterpret_cast<int*>(mm + 4);
  if (nocc > 0 && naux > 0 && have_tgam) {
    GemmDesc g;  // Drec = 2 Ct^T Ct
    g.M = n; g.N = n; g.K = nocc;
    g.A = Ct; g.lda = n; g.opA = Op::T;
    g.B = Ct; g.ldb = n; g.C = Drec; g.ldc = n; g.alpha = 2.0;
    gemm(g, s);
    RR_CUDA(cudaMemsetAsync(mm, 0, 2 * sizeof(double), s));
    density_diff_kernel<<<static_cast<int>(std::min<int64_t>((n2 + 255) / 256, 296)), 256, 0, s>>>(Dp, Drec, n2, mm);
    RR_LAUNCH_CHECK();
    density_flag_kernel<<<1, 1, 0, s>>>(mm, flag);
    RR_LAUNCH_CHECK();
  } else {
    RR_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
  }
  auto& jp = h->jpend;
  jp.pl = pl;
  jp.gpart = h->jscr.p;
  jp.jpart = h->jscr.p + goff;
  jp.flag = flag;
  jp.s = s;
  jp.overlap = overlap;
}

// s_in: the stream that ran the half-transform (the one coulomb_prep was given).
void coulomb_run(rr_ri_store* h, const double* tgam, int tseg, cudaStream_t s_in) {
  auto& c = h->ctx;
  auto& jp = h->jpend;
  const cudaStream_t s = jp.s;
  if (jp.overlap) {
    RR_CUDA(cudaEventRecord(c.mid, s_in));
    RR_CUDA(cudaStreamWaitEvent(s, c.mid, 0));
  }
  prof_mark(h, 5, s);  // J phase = the passes (the preparation overlaps the half-transform)
  j_pass1(jp.pl, jp.gpart, h->status.p, s, jp.flag);
  j_pass2(jp.pl, jp.gpart, jp.jpart, h->status.p, s, tgam, tseg, jp.flag);
  j_finish(jp.pl, jp.jpart, 1.0, s);
  prof_mark(h, 6, s);
  RR_CUDA(cudaEventRecord(c.join, s));  // without overlap coulomb_join is a no-op wait on the same stream
}

void coulomb_after_ht(rr_ri_store* h, const double* Dp, const double* Ct, int64_t nocc, double* J,
                      const double* tgam, int tseg, cudaStream_t s) {
  coulomb_prep(h, Dp, Ct, nocc, J, tgam != nullptr, s, false);
  coulomb_run(h, tgam, tseg, s);
}

// Both J passes from the density alone, on the side stream from the current point of s: the
// drop-in build starts them before the occupied recovery, whose small products leave most of the
// GPU idle.  Join with coulomb_join.
void coulomb_early(rr_ri_store* h, const double* Dp, double* J, cudaStream_t s, int ctas_per_sm) {
  const int64_t n = h->n, naux = h->naux;
  auto& c = h->ctx;
  RR_CUDA(cudaEventRecord(c.fork, s));
  RR_CUDA(cudaStreamWaitEvent(c.side, c.fork, 0));
  h->dfold.ensure(static_cast<size_t>(tri_len(n) + 1));
  JTensor t = j_tensor(h, 0, n, Dp, J, 0, c.side);
  JPlan pl = j_plan(1, &t, naux, ctas_per_sm);
  const int64_t goff = round_up(pl.gpart_doubles, 32);
  h->jscr.ensure(static_cast<size_t>(goff + pl.jpart_doubles + 32));
  prof_mark(h, 5, c.side);
  j_pass1(pl, h->jscr.p, h->status.p, c.side);
  j_pass2(pl, h->jscr.p, h->jscr.p + goff, h->status.p, c.side);
  j_finish(pl, h->jscr.p + goff, 1.0, c.side);
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
  cudaEvent_t d_ready = nullptr, h_ready = nullptr;
  if (host) {
    // Host inputs arrive on the side stream in the order they are read: S and X (the recovery's
    // first product is S X), then D (then the J passes and h, below), so the later copies overlap
    // the recovery.
    auto& c = h->ctx;
    RR_CUDA(cudaEventRecord(c.fork, s));
    RR_CUDA(cudaStreamWaitEvent(c.side, c.fork, 0));
    copy_in(Sd, S, n2, true, c.side);
    copy_in(Xd, X, n * n_eff, true, c.side);
    RR_CUDA(cudaEventRecord(c.upl[0], c.side));
    copy_in_padded(Dp, pitch, D, n2, true, c.side);
    RR_CUDA(cudaEventRecord(c.upl[1], c.side));
    RR_CUDA(cudaStreamWaitEvent(s, c.upl[0], 0));
    d_ready = c.upl[1];
  } else {
    copy_in_padded(Dp, pitch, D, n2, false, s);
  }
  // J from the density on the side stream (after the upload of D there), beside the occupied
  // recovery (X^T (S D S / 2) X, eigenvalues > 0.5) as c_t = F^T X^T on s, then the exchange.
  // One J CTA per SM: it shares the SMs with the recovery and then the half-transform (measured at
  // n = 400, naux = 1600, nocc = 40: 1.67 ms per build with one, 1.70 with two, 1.81 with three);
  // RR_J_CTAS=<k> sets another count for measurement.
  static const int j_ctas = [] {
    const char* e = std::getenv("RR_J_CTAS");
    const int k = e ? std::atoi(e) : 1;
    return k >= 1 && k <= 4 ? k : 1;
  }();
  // RR_J_AFTER_RECOVERY=1 (device pointers, for measurement): the J passes start after the recovery
  // instead, beside the half-transform and the SYRK only: 1.630 / 1.748 / 1.818 ms per build with 1 / 2 / 3
  // J CTAs per SM, against 1.565 / 1.584 / 1.708 ms from the top of the build.
  static const bool j_late = [] {
    const char* e = std::getenv("RR_J_AFTER_RECOVERY");
    return e && std::atoi(e) == 1;
  }();
  if (host) {
    auto& c = h->ctx;
    coulomb_early(h, Dp, J, c.side, j_ctas);
    copy_in(hd, hc, n2, true, c.side);  // read only by the final combine
    RR_CUDA(cudaEventRecord(c.upl[2], c.side));
    h_ready = c.upl[2];
  } else if (!j_late) {
    coulomb_early(h, Dp, J, s, j_ctas);
  }
  const int64_t nocc = occupied_ct(h, Xd, Sd, Dp, n, n_eff, 0.5, false, false, Ct, s, d_ready);
  if (!host && j_late) coulomb_early(h, Dp, J, s, j_ctas);
  if (d_ready) RR_CUDA(cudaStreamWaitEvent(s, d_ready, 0));  // (n_eff = 0 skips the products)
  prof_mark(h, 1, s);
  exchange_nonrel(h, Ct, n, false, nocc, K, s);
  prof_mark(h, 3, s);
  coulomb_join(h, s);
  if (h_ready) RR_CUDA(cudaStreamWaitEvent(s, h_ready, 0));
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
  double *Dp, *Cd, *J, *K, *Ctj;
  Arena ar(&h->mats);
  ar.request(&Dp, pitch);
  ar.request(&Ctj, std::max<int64_t>(nocc, 1) * n);
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
  prof_mark(h, 1, s);
  transpose(Ctj, Cd, n, nocc, s);  // c_t = C^T, row-major nocc x n
  if (o && o->precision == RR_PREC_MIXED) {
    // Split-BF16 exchange on tcgen05; Coulomb in FP64 (two streaming passes over B).
    mixed_prepare(h->mixed[0], h->B[0].p, h->pitch[0], n, h->naux, s);
    prof_mark(h, 2, s);
    mixed_exchange(h->mixed[0], h->mscr, Ctj, n, nocc, K, h->status.p, s);
    coulomb_after_ht(h, Dp, Ctj, 0, J, nullptr, 0, s);
  } else {
    exchange_nonrel(h, Ctj, n, false, nocc, K, s, Dp, J);
  }
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
