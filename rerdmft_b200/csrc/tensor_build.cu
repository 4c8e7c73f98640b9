// One-time set-up of the RI tensor on the device: the reference's canonical (LOWGEN) orthogonalisation,
// the metric contraction B = X_metric^T raw and the per-aux-row AO-leg transform t^T B^P t.
//
// Reference: canonicalOrthogonalize / canonicalOrthogonalizeHermitian
// (src/Linear_Algebra/LinearAlgebra.cpp:267-349; used for the AO overlaps under X_LIN_DEP_THRS_L/S,
// main.cpp:4476, 4544, 4584, and for the aux metric, src/AO_ints/ThreeCenterIntegrals.cpp:185-189),
// riThreeCenterTensor's contraction (ThreeCenterIntegrals.cpp:219-236) and transformRiThreeCenterAoLegs
// (:191-217).  The raw 3-centre integrals themselves come from libcint on the host, as in the reference.
//
// These run once per basis, so they use a private stream, a private cuSOLVER handle and scratch
// allocated per call.
#include <algorithm>
#include <cmath>
#include <vector>

#include "ri_store.cuh"

namespace rr {

namespace {

int blocks_for(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 1184))); }

// A = D^-1 S D^-1 with D = diag(sqrt(Re S_ii)) (interleaved complex): the Jacobi scaling of
// canonicalOrthogonalizeHermitian (LinearAlgebra.cpp:322-327).
__global__ void jacobi_scale_kernel(double* A, const double* S, int64_t n) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < n * n;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx / n, j = idx % n;
    const double f = 1.0 / (sqrt(S[2 * (i * n + i)]) * sqrt(S[2 * (j * n + j)]));
    A[2 * idx] = S[2 * idx] * f;
    A[2 * idx + 1] = S[2 * idx + 1] * f;
  }
}

// X(i, j) = U(i, k0 + j) / sqrt(w[k0 + j]) (/ d_i when S is given, the Hermitian version), X: n x n_eff.
// Row k of Urows holds eigenvector k (conjugated for the complex solver, which sees the row-major
// matrix as its transpose): U(i, k) = Urows[k][i] (real) or conj(Urows[k][i]) (complex).
template <int PL>
__global__ void orth_columns_kernel(const double* Urows, const double* w, int64_t n, int64_t k0, int64_t n_eff,
                                    const double* S, double* X) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < n * n_eff;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx / n_eff, j = idx % n_eff, k = k0 + j;
    double fac = 1.0 / sqrt(w[k]);
    if (S) fac /= sqrt(S[PL * (i * n + i)]);
    const int64_t src = k * n + i;
    X[PL * idx] = Urows[PL * src] * fac;
    if (PL == 2) X[2 * idx + 1] = -Urows[2 * src + 1] * fac;
  }
}

// Private stream and cuSOLVER handle of a handle-free set-up call.
struct SetupCtx {
  cudaStream_t s = nullptr;
  bool own = false;
  cusolverDnHandle_t solver = nullptr;
  explicit SetupCtx(const rr_opts* o) {
    if (o && o->stream) {
      s = static_cast<cudaStream_t>(o->stream);
    } else {
      RR_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      own = true;
    }
  }
  cusolverDnHandle_t get_solver() {
    if (!solver) {
      RR_SOLVER(cusolverDnCreate(&solver));
      RR_SOLVER(cusolverDnSetStream(solver, s));
    }
    return solver;
  }
  ~SetupCtx() {
    if (solver) cusolverDnDestroy(solver);
    if (own && s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
};

bool is_host(const rr_opts* o) { return !o || o->mem == RR_MEM_HOST; }

// Device view of a caller's matrix: the pointer itself (device memory) or an uploaded copy.
const double* device_view(const double* p, int64_t count, bool host, DevBuf<double>& tmp, cudaStream_t s) {
  if (!host || count <= 0) return p;
  tmp.alloc(static_cast<size_t>(count));
  RR_CUDA(cudaMemcpyAsync(tmp.p, p, sizeof(double) * count, cudaMemcpyHostToDevice, s));
  return tmp.p;
}

// Symmetric / Hermitian eigensolver on the device (cuSOLVER syevd / heevd) in place on row-major A:
// row k becomes eigenvector k (conjugated when complex), w ascending.  Throws on a solver failure.
void eigh_inplace(SetupCtx& c, double* A, int64_t n, double* w, bool cplx) {
  cusolverDnHandle_t sv = c.get_solver();
  int lwork = 0;
  DevBuf<int> info(1);
  DevBuf<double> work;
  if (cplx) {
    auto* az = reinterpret_cast<cuDoubleComplex*>(A);
    RR_SOLVER(cusolverDnZheevd_bufferSize(sv, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, static_cast<int>(n), az,
                                          static_cast<int>(n), w, &lwork));
    work.alloc(2 * static_cast<size_t>(lwork) + 2);
    RR_SOLVER(cusolverDnZheevd(sv, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, static_cast<int>(n), az,
                               static_cast<int>(n), w, reinterpret_cast<cuDoubleComplex*>(work.p), lwork, info.p));
  } else {
    RR_SOLVER(cusolverDnDsyevd_bufferSize(sv, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, static_cast<int>(n), A,
                                          static_cast<int>(n), w, &lwork));
    work.alloc(static_cast<size_t>(lwork) + 1);
    RR_SOLVER(cusolverDnDsyevd(sv, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, static_cast<int>(n), A,
                               static_cast<int>(n), w, work.p, lwork, info.p));
  }
  int hinfo = 0;
  RR_CUDA(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, c.s));
  RR_CUDA(cudaStreamSynchronize(c.s));
  RR_REQUIRE(hinfo == 0, RR_ERR_SOLVER, "diagonalize: the eigensolver did not converge (info " + std::to_string(hinfo) + ")");
}

}  // namespace

void canonical_orthogonalize(const double* S, int64_t n, bool herm, double threshold, double* X, int64_t* n_eff_out,
                             rr_rank_report* report, const rr_opts* o) {
  const bool host = is_host(o);
  SetupCtx c(o);
  const int PL = herm ? 2 : 1;
  DevBuf<double> Sup, A(static_cast<size_t>(n * n * PL)), w(static_cast<size_t>(n)), Xd(static_cast<size_t>(n * n * PL));
  const double* Sd = device_view(S, n * n * PL, host, Sup, c.s);
  if (herm) {
    jacobi_scale_kernel<<<blocks_for(n * n), 256, 0, c.s>>>(A.p, Sd, n);
    RR_LAUNCH_CHECK();
  } else {
    RR_CUDA(cudaMemcpyAsync(A.p, Sd, sizeof(double) * n * n, cudaMemcpyDeviceToDevice, c.s));
  }
  eigh_inplace(c, A.p, n, w.p, herm);
  std::vector<double> wh(static_cast<size_t>(n));
  RR_CUDA(cudaMemcpyAsync(wh.data(), w.p, sizeof(double) * n, cudaMemcpyDeviceToHost, c.s));
  RR_CUDA(cudaStreamSynchronize(c.s));
  // keep the eigenvalues above the threshold (a suffix of the ascending list), with the reference's
  // report fields (LinearAlgebra.cpp:271-280: smallest kept, largest dropped, both 0 when empty)
  int64_t k0 = n;
  for (int64_t i = 0; i < n; ++i)
    if (wh[i] > threshold) {
      k0 = i;
      break;
    }
  for (int64_t i = k0; i < n; ++i)
    RR_REQUIRE(wh[i] > threshold, RR_ERR_SOLVER, "canonicalOrthogonalize: eigenvalues not in ascending order");
  const int64_t n_eff = n - k0;
  double largest_dropped = 0.0;
  for (int64_t i = 0; i < k0; ++i) largest_dropped = std::max(largest_dropped, wh[i]);
  if (report) {
    report->n_kept = n_eff;
    report->n_dropped = k0;
    report->smallest_kept = n_eff > 0 ? wh[k0] : 0.0;
    report->largest_dropped = largest_dropped;
  }
  *n_eff_out = n_eff;
  if (n_eff > 0) {
    if (herm)
      orth_columns_kernel<2><<<blocks_for(n * n_eff), 256, 0, c.s>>>(A.p, w.p, n, k0, n_eff, Sd, Xd.p);
    else
      orth_columns_kernel<1><<<blocks_for(n * n_eff), 256, 0, c.s>>>(A.p, w.p, n, k0, n_eff, nullptr, Xd.p);
    RR_LAUNCH_CHECK();
    const double* Xout = Xd.p;
    DevBuf<double> Xs;
    if (!herm && n_eff == n) {
      // nothing dropped: X U^T, the symmetric S^-1/2 (LinearAlgebra.cpp:303-309); U^T = A's rows
      Xs.alloc(static_cast<size_t>(n * n));
      GemmDesc g;
      g.M = n; g.N = n; g.K = n; g.A = Xd.p; g.lda = n; g.B = A.p; g.ldb = n; g.C = Xs.p; g.ldc = n;
      gemm(g, c.s);
      Xout = Xs.p;
    }
    RR_CUDA(cudaMemcpyAsync(X, Xout, sizeof(double) * n * n_eff * PL,
                            host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, c.s));
  }
  RR_CUDA(cudaStreamSynchronize(c.s));
}

// B (naux_kept x n2, row pitch ldb) = metric_x^T raw, metric_x: naux_raw x naux_kept, raw: naux_raw x n2
// (device pointers).
void metric_contract(const double* raw, int64_t naux_raw, int64_t n2, const double* mx, int64_t naux_kept, double* B,
                     int64_t ldb, cudaStream_t s) {
  GemmDesc g;
  g.M = naux_kept; g.N = n2; g.K = naux_raw;
  g.A = mx; g.lda = naux_kept; g.opA = Op::T;
  g.B = raw; g.ldb = n2;
  g.C = B; g.ldc = ldb;
  gemm(g, s);
}

// out^P (n_out x n_out, row pitch ld_out per aux row) = t^T B^P t for P < naux; B^P is n_ao x n_ao with
// row pitch ld_in per aux row; t: n_ao x n_out (device pointers).  The intermediate t^T B^P is held for
// at most 32M doubles of aux rows at a time.
void ao_leg_transform(const double* B, int64_t ld_in, int64_t naux, int64_t n_ao, const double* t, int64_t n_out,
                      double* out, int64_t ld_out, cudaStream_t s) {
  if (naux == 0 || n_out == 0) return;
  const int64_t per = std::max<int64_t>(1, n_out * n_ao);
  const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(naux, (32LL << 20) / per));
  DevBuf<double> U(static_cast<size_t>(chunk * per));
  for (int64_t p0 = 0; p0 < naux; p0 += chunk) {
    const int64_t nb = std::min(chunk, naux - p0);
    GemmDesc a;  // U_P = t^T B^P
    a.M = n_out; a.N = n_ao; a.K = n_ao;
    a.A = t; a.lda = n_out; a.opA = Op::T; a.strideA = 0;
    a.B = B + p0 * ld_in; a.ldb = n_ao; a.strideB = ld_in;
    a.C = U.p; a.ldc = n_ao; a.strideC = per;
    a.batch = nb;
    gemm(a, s);
    GemmDesc b;  // out_P = U_P t
    b.M = n_out; b.N = n_out; b.K = n_ao;
    b.A = U.p; b.lda = n_ao; b.strideA = per;
    b.B = t; b.ldb = n_out; b.strideB = 0;
    b.C = out + p0 * ld_out; b.ldc = n_out; b.strideC = ld_out;
    b.batch = nb;
    gemm(b, s);
  }
}

}  // namespace rr

namespace {

template <typename F>
int setup_api(F&& f) {
  try {
    rr::set_last_error("");
    f();
    return RR_OK;
  } catch (const rr::Error& e) {
    rr::set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    rr::set_last_error("host allocation failed");
    return RR_ERR_NOMEM;
  } catch (const std::exception& e) {
    rr::set_last_error(e.what());
    return RR_ERR_CUDA;
  }
}

}  // namespace

extern "C" {

int rr_canonical_orthogonalize(const double* S, int64_t n, int32_t hermitian, double threshold, double* X,
                               int64_t* n_eff, rr_rank_report* report, const rr_opts* opts) {
  return setup_api([&] {
    RR_REQUIRE(n >= 1 && S && X && n_eff, RR_ERR_ARG, "canonicalOrthogonalize: need n >= 1 and non-null S, X, n_eff");
    RR_REQUIRE(!opts || opts->precision == RR_PREC_FP64, RR_ERR_UNSUPPORTED, "canonicalOrthogonalize: precision");
    rr::canonical_orthogonalize(S, n, hermitian != 0, threshold, X, n_eff, report, opts);
  });
}

int rr_ri_three_center_tensor(const double* raw, int64_t naux_raw, int64_t n2, const double* metric_x,
                              int64_t naux_kept, double* B, const rr_opts* opts) {
  return setup_api([&] {
    RR_REQUIRE(naux_raw >= 0 && n2 >= 0 && naux_kept >= 0, RR_ERR_ARG, "riThreeCenterTensor: negative size");
    RR_REQUIRE((raw && metric_x && B) || naux_kept * n2 == 0, RR_ERR_ARG, "riThreeCenterTensor: null matrix");
    if (naux_kept * n2 == 0) return;
    const bool host = rr::is_host(opts);
    rr::SetupCtx c(opts);
    rr::DevBuf<double> ru, mu, bo;
    const double* rd = rr::device_view(raw, naux_raw * n2, host, ru, c.s);
    const double* md = rr::device_view(metric_x, naux_raw * naux_kept, host, mu, c.s);
    double* bd = B;
    if (host) {
      bo.alloc(static_cast<size_t>(naux_kept * n2));
      bd = bo.p;
    }
    rr::metric_contract(rd, naux_raw, n2, md, naux_kept, bd, n2, c.s);
    if (host) RR_CUDA(cudaMemcpyAsync(B, bd, sizeof(double) * naux_kept * n2, cudaMemcpyDeviceToHost, c.s));
    RR_CUDA(cudaStreamSynchronize(c.s));
  });
}

int rr_ri_transform_ao_legs(const double* B_in, int64_t naux, int64_t n_ao, const double* t, int64_t n_out,
                            double* B_out, const rr_opts* opts) {
  return setup_api([&] {
    RR_REQUIRE(naux >= 0 && n_ao >= 0 && n_out >= 0, RR_ERR_ARG, "transformRiThreeCenterAoLegs: negative size");
    if (naux == 0 || n_out == 0) return;
    RR_REQUIRE(B_in && t && B_out, RR_ERR_ARG, "transformRiThreeCenterAoLegs: null matrix");
    const bool host = rr::is_host(opts);
    rr::SetupCtx c(opts);
    const int64_t cnt_out = naux * n_out * n_out;
    if (n_ao == 0) {  // the reference returns zeros
      if (host) std::fill(B_out, B_out + cnt_out, 0.0);
      else RR_CUDA(cudaMemsetAsync(B_out, 0, sizeof(double) * cnt_out, c.s));
      RR_CUDA(cudaStreamSynchronize(c.s));
      return;
    }
    rr::DevBuf<double> bu, tu, bo;
    const double* bd = rr::device_view(B_in, naux * n_ao * n_ao, host, bu, c.s);
    const double* td = rr::device_view(t, n_ao * n_out, host, tu, c.s);
    double* od = B_out;
    if (host) {
      bo.alloc(static_cast<size_t>(cnt_out));
      od = bo.p;
    }
    rr::ao_leg_transform(bd, n_ao * n_ao, naux, n_ao, td, n_out, od, n_out * n_out, c.s);
    if (host) RR_CUDA(cudaMemcpyAsync(B_out, od, sizeof(double) * cnt_out, cudaMemcpyDeviceToHost, c.s));
    RR_CUDA(cudaStreamSynchronize(c.s));
  });
}

int rr_ri_create_raw(const double* raw, int64_t naux_raw, int64_t n_ao, const double* metric_x, int64_t naux_kept,
                     const double* t, int64_t n_out, int32_t mem, rr_ri_handle* out) {
  return setup_api([&] {
    RR_REQUIRE(out != nullptr, RR_ERR_ARG, "rr_ri_create_raw: out is null");
    *out = nullptr;
    RR_REQUIRE(naux_raw >= 0 && naux_kept >= 0 && n_ao >= 1, RR_ERR_ARG, "rr_ri_create_raw: bad dimensions");
    RR_REQUIRE(mem == RR_MEM_HOST || mem == RR_MEM_DEVICE, RR_ERR_ARG, "rr_ri_create_raw: bad mem kind");
    if (!t) n_out = n_ao;
    RR_REQUIRE(n_out >= 1, RR_ERR_ARG, "rr_ri_create_raw: n_out must be >= 1");
    RR_REQUIRE((raw && metric_x) || naux_kept == 0, RR_ERR_ARG, "rr_ri_create_raw: null matrix");
    const bool host = mem == RR_MEM_HOST;
    auto* h = new rr_ri_store();
    try {
      h->ctx.init(nullptr);
      cudaStream_t s = h->ctx.main;
      h->naux = naux_kept;
      h->n = n_out;
      h->ntens = 1;
      h->status.alloc(2);
      RR_CUDA(cudaMemsetAsync(h->status.p, 0, 2 * sizeof(int), s));
      const int64_t n2o = n_out * n_out, n2a = n_ao * n_ao;
      h->pitch[0] = rr::round_up(std::max<int64_t>(n2o, 2), 32);
      h->B[0].alloc(static_cast<size_t>(std::max<int64_t>(naux_kept * h->pitch[0], 32)));
      RR_CUDA(cudaMemsetAsync(h->B[0].p, 0, sizeof(double) * h->B[0].n, s));
      if (naux_kept > 0) {
        rr::DevBuf<double> ru, mu, tu, full;
        const double* rd = rr::device_view(raw, naux_raw * n2a, host, ru, s);
        const double* md = rr::device_view(metric_x, naux_raw * naux_kept, host, mu, s);
        if (t) {
          // the reference's order: the metric contraction of the raw tensor, then the AO legs
          const double* td = rr::device_view(t, n_ao * n_out, host, tu, s);
          full.alloc(static_cast<size_t>(naux_kept * n2a));
          rr::metric_contract(rd, naux_raw, n2a, md, naux_kept, full.p, n2a, s);
          rr::ao_leg_transform(full.p, n2a, naux_kept, n_ao, td, n_out, h->B[0].p, h->pitch[0], s);
        } else {
          rr::metric_contract(rd, naux_raw, n2a, md, naux_kept, h->B[0].p, h->pitch[0], s);
        }
        RR_CUDA(cudaStreamSynchronize(s));
      }
      rr::pack_for_j(h, 0, n_out, s);
      RR_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
      h->ctx.destroy();
      delete h;
      throw;
    }
    *out = h;
  });
}

}  // extern "C"
