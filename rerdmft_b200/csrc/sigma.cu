// RI sigma-vector Hessian-vector primitives on the device: the GEMM engine behind the NEO optimiser's
// orbital-rotation Hessian-vector products.
//
// Reference: src/Hessian_opt/RiSigmaHessianToolkit.cpp:24-55 (buildRiSigmaHessianToolkit: KB1[P] =
// K B^P, KB2[P] = B^P K and three diagonals) and src/Hessian_opt/RiSigmaGemm.cpp:65-126 (pairContract,
// diagContract, accumU).  The tensors are (naux, n^2) row-major, real or interleaved complex; K, w,
// post and Wm are real and multiply the complex operands unconjugated, as in the reference.
//
//   pairContract:  target(x,y) += sign sum_{P,t} F(P,t,x) G(P,t,y): each operand is gathered into a
//                  (naux n) x n matrix by one kernel (and right-multiplied by `post` on the tensor
//                  cores when given), then one DMMA GEMM F^T G with a split K of naux n.
//   diagContract:  target(a,b) += sum_P S(P, b n + a) (Ua(P,a) + Ub(P,b)), one thread per (a, b).
//   accumU:        U += alpha D Wm^T, one GEMM.
#include <algorithm>

#include "ri_store.cuh"

namespace rr {
namespace {

int blocks_for(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4736))); }

template <int PL>
__device__ __forceinline__ void cmul(double& re, double& im, double br, double bi) {
  if (PL == 2) {
    const double r = re * br - im * bi;
    im = re * bi + im * br;
    re = r;
  } else {
    re *= br;
  }
}

// dst[(P n + t) n + x] = s(P, idx[t n + x]) * w[t n + x] * row(P, t) (each factor 1 when absent).
template <int PL>
__global__ void pair_fill_kernel(double* dst, const double* s, const uint32_t* idx, const double* w, const double* row,
                                 int64_t n, int64_t naux) {
  const int64_t n2 = n * n, total = naux * n2;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t P = e / n2, tx = e % n2, t = tx / n;
    double re = 1.0, im = 0.0;
    if (s) {
      const int64_t src = P * n2 + idx[tx];
      re = s[PL * src];
      if (PL == 2) im = s[2 * src + 1];
    }
    if (w) {
      re *= w[tx];
      im *= w[tx];
    }
    if (row) cmul<PL>(re, im, row[PL * (P * n + t)], PL == 2 ? row[2 * (P * n + t) + 1] : 0.0);
    dst[PL * e] = re;
    if (PL == 2) dst[2 * e + 1] = im;
  }
}

// target(a, b) += sum_P S(P, b n + a) (Ua(P, a) + Ub(P, b)).
template <int PL>
__global__ void diag_contract_kernel(double* target, const double* S, const double* Ua, const double* Ub, int64_t n,
                                     int64_t naux) {
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n * n;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t b = e / n, a = e % n;  // consecutive threads: consecutive a, contiguous S
    double ar = 0.0, ai = 0.0;
    for (int64_t P = 0; P < naux; ++P) {
      double ur = 0.0, ui = 0.0;
      if (Ua) { ur += Ua[PL * (P * n + a)]; if (PL == 2) ui += Ua[2 * (P * n + a) + 1]; }
      if (Ub) { ur += Ub[PL * (P * n + b)]; if (PL == 2) ui += Ub[2 * (P * n + b) + 1]; }
      const int64_t si = P * n * n + b * n + a;
      const double sr = S[PL * si], sim = PL == 2 ? S[2 * si + 1] : 0.0;
      ar += sr * ur - sim * ui;
      if (PL == 2) ai += sr * ui + sim * ur;
    }
    double* t = target + PL * (a * n + b);
    t[0] += ar;
    if (PL == 2) t[1] += ai;
  }
}

// out (interleaved complex, n2 entries) = real in.
__global__ void complexify_kernel(double* out, const double* in, int64_t n2) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n2;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    out[2 * i] = in[i];
    out[2 * i + 1] = 0.0;
  }
}

// diag[P n + x] = M(P, x n + x) for each of `cnt` tensors.
template <int PL>
__global__ void diagonals_kernel(const double* M, double* diag, int64_t n, int64_t naux) {
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < naux * n;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t P = e / n, x = e % n, src = P * n * n + x * n + x;
    diag[PL * e] = M[PL * src];
    if (PL == 2) diag[2 * e + 1] = M[2 * src + 1];
  }
}

struct SigmaCtx {
  cudaStream_t s = nullptr;
  bool own = false, host = true;
  explicit SigmaCtx(const rr_opts* o) {
    host = !o || o->mem == RR_MEM_HOST;
    if (o && o->stream) {
      s = static_cast<cudaStream_t>(o->stream);
    } else {
      RR_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      own = true;
    }
  }
  // Device view of a caller's input (uploaded when the call has host pointers).
  template <typename T>
  const T* in(const T* p, int64_t count, DevBuf<T>& tmp) {
    if (!host || !p || count <= 0) return p;
    tmp.alloc(static_cast<size_t>(count));
    RR_CUDA(cudaMemcpyAsync(tmp.p, p, sizeof(T) * count, cudaMemcpyHostToDevice, s));
    return tmp.p;
  }
  // Device buffer for an in/out argument (uploaded for host calls; written back by out()).
  double* inout(double* p, int64_t count, DevBuf<double>& tmp) {
    if (!host) return p;
    tmp.alloc(static_cast<size_t>(std::max<int64_t>(count, 1)));
    RR_CUDA(cudaMemcpyAsync(tmp.p, p, sizeof(double) * count, cudaMemcpyHostToDevice, s));
    return tmp.p;
  }
  void out(double* host_p, const double* dev_p, int64_t count) {
    if (host && count > 0) RR_CUDA(cudaMemcpyAsync(host_p, dev_p, sizeof(double) * count, cudaMemcpyDeviceToHost, s));
  }
  void finish(const rr_opts* o) {
    if (host || own || (o && o->sync)) RR_CUDA(cudaStreamSynchronize(s));
  }
  ~SigmaCtx() {
    if (own && s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
};

// The real n x n matrix m as the operand of a product with PL-plane values (complexified for PL = 2).
const double* real_operand(const double* m, int64_t n, bool cplx, DevBuf<double>& tmp, cudaStream_t s) {
  if (!cplx) return m;
  tmp.alloc(static_cast<size_t>(2 * n * n));
  complexify_kernel<<<blocks_for(n * n), 256, 0, s>>>(tmp.p, m, n * n);
  RR_LAUNCH_CHECK();
  return tmp.p;
}

// Operand values of one PairOp into dst ((naux n) x n, PL planes): gather, then `post` when given.
void pair_operand(const rr_pair_op& op, int64_t n, int64_t naux, bool cplx, SigmaCtx& c, double* dst,
                  DevBuf<double>& scratch, DevBuf<double> (&tmp)[5], DevBuf<uint32_t>& itmp) {
  const int PL = cplx ? 2 : 1;
  const int64_t n2 = n * n;
  const double* s = c.in(op.s, naux * n2 * PL, tmp[0]);
  const uint32_t* idx = op.s ? c.in(op.idx, n2, itmp) : nullptr;
  const double* w = c.in(op.w, n2, tmp[1]);
  const double* row = c.in(op.row, naux * n * PL, tmp[2]);
  double* out = dst;
  if (op.post) {
    scratch.ensure(static_cast<size_t>(naux * n2 * PL));
    out = scratch.p;
  }
  if (cplx) pair_fill_kernel<2><<<blocks_for(naux * n2), 256, 0, c.s>>>(out, s, idx, w, row, n, naux);
  else pair_fill_kernel<1><<<blocks_for(naux * n2), 256, 0, c.s>>>(out, s, idx, w, row, n, naux);
  RR_LAUNCH_CHECK();
  if (op.post) {
    const double* post = real_operand(c.in(op.post, n2, tmp[3]), n, cplx, tmp[4], c.s);
    GemmDesc g;  // dst = values * post
    g.cplx = cplx;
    g.M = naux * n; g.N = n; g.K = n;
    g.A = out; g.lda = n; g.B = post; g.ldb = n; g.C = dst; g.ldc = n;
    gemm(g, c.s);
  }
}

}  // namespace
}  // namespace rr

namespace {

template <typename F>
int sigma_api(F&& f) {
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

int rr_sigma_toolkit(const double* B, int64_t n, int64_t naux, int32_t cplx, const double* K, double* kb1, double* kb2,
                     double* bdiag, double* kb1diag, double* kb2diag, const rr_opts* opts) {
  return sigma_api([&] {
    RR_REQUIRE(n >= 0 && naux >= 0, RR_ERR_ARG, "buildRiSigmaHessianToolkit: negative size");
    RR_REQUIRE((B && K && kb1 && kb2 && bdiag && kb1diag && kb2diag) || n * naux == 0, RR_ERR_ARG,
               "buildRiSigmaHessianToolkit: null matrix");
    if (n * naux == 0) return;
    const int PL = cplx ? 2 : 1;
    const int64_t n2 = n * n, tot = naux * n2 * PL, dtot = naux * n * PL;
    rr::SigmaCtx c(opts);
    rr::DevBuf<double> tb, tk, kc, o1, o2, d0, d1, d2;
    const double* Bd = c.in(B, tot, tb);
    const double* Kd = rr::real_operand(c.in(K, n2, tk), n, cplx != 0, kc, c.s);
    double* k1 = c.host ? (o1.alloc(static_cast<size_t>(tot)), o1.p) : kb1;
    double* k2 = c.host ? (o2.alloc(static_cast<size_t>(tot)), o2.p) : kb2;
    rr::GemmDesc g;  // KB1[P] = K B^P
    g.cplx = cplx != 0;
    g.M = n; g.N = n; g.K = n; g.batch = naux;
    g.A = Kd; g.lda = n; g.strideA = 0;
    g.B = Bd; g.ldb = n; g.strideB = n2;
    g.C = k1; g.ldc = n; g.strideC = n2;
    rr::gemm(g, c.s);
    g.A = Bd; g.strideA = n2;  // KB2[P] = B^P K
    g.B = Kd; g.strideB = 0;
    g.C = k2;
    rr::gemm(g, c.s);
    double* dd[3] = {c.host ? (d0.alloc(static_cast<size_t>(dtot)), d0.p) : bdiag,
                     c.host ? (d1.alloc(static_cast<size_t>(dtot)), d1.p) : kb1diag,
                     c.host ? (d2.alloc(static_cast<size_t>(dtot)), d2.p) : kb2diag};
    const double* src[3] = {Bd, k1, k2};
    for (int i = 0; i < 3; ++i) {
      if (cplx) rr::diagonals_kernel<2><<<rr::blocks_for(naux * n), 256, 0, c.s>>>(src[i], dd[i], n, naux);
      else rr::diagonals_kernel<1><<<rr::blocks_for(naux * n), 256, 0, c.s>>>(src[i], dd[i], n, naux);
      RR_LAUNCH_CHECK();
    }
    c.out(kb1, k1, tot);
    c.out(kb2, k2, tot);
    c.out(bdiag, dd[0], dtot);
    c.out(kb1diag, dd[1], dtot);
    c.out(kb2diag, dd[2], dtot);
    c.finish(opts);
  });
}

int rr_sigma_pair_contract(double* target, double sign, int64_t n, int64_t naux, int32_t cplx, const rr_pair_op* f,
                           const rr_pair_op* g, const rr_opts* opts) {
  return sigma_api([&] {
    RR_REQUIRE(target && f && g && n >= 0 && naux >= 0, RR_ERR_ARG, "pairContract: bad arguments");
    RR_REQUIRE((!f->s || f->idx) && (!g->s || g->idx), RR_ERR_ARG, "pairContract: an operand with s needs idx");
    if (n == 0 || naux == 0) return;  // the reference returns without touching target
    const int PL = cplx ? 2 : 1;
    const int64_t rows = naux * n, cnt = rows * n * PL;
    rr::SigmaCtx c(opts);
    rr::DevBuf<double> fb(static_cast<size_t>(cnt)), gb(static_cast<size_t>(cnt)), scratch, tt, tmpf[5], tmpg[5];
    rr::DevBuf<uint32_t> itf, itg;
    rr::pair_operand(*f, n, naux, cplx != 0, c, fb.p, scratch, tmpf, itf);
    rr::pair_operand(*g, n, naux, cplx != 0, c, gb.p, scratch, tmpg, itg);
    double* T = c.inout(target, n * n * PL, tt);
    rr::GemmDesc m;  // target += sign F^T G over the naux n rows
    m.cplx = cplx != 0;
    m.M = n; m.N = n; m.K = rows;
    m.A = fb.p; m.lda = n; m.opA = rr::Op::T;
    m.B = gb.p; m.ldb = n;
    m.C = T; m.ldc = n;
    m.alpha = sign; m.beta = 1.0;
    rr::DevBuf<double> work(static_cast<size_t>(std::max<int64_t>(rr::gemm_work_doubles(m), 1)));
    rr::gemm(m, c.s, work.p, static_cast<int64_t>(work.n));
    c.out(target, T, n * n * PL);
    c.finish(opts);
  });
}

int rr_sigma_diag_contract(double* target, int64_t n, int64_t naux, int32_t cplx, const double* S, const double* Ua,
                           const double* Ub, const rr_opts* opts) {
  return sigma_api([&] {
    RR_REQUIRE(target && (S || n * naux == 0) && n >= 0 && naux >= 0, RR_ERR_ARG, "diagContract: bad arguments");
    if (n == 0) return;
    const int PL = cplx ? 2 : 1;
    rr::SigmaCtx c(opts);
    rr::DevBuf<double> ts, ta, tb, tt;
    const double* Sd = c.in(S, naux * n * n * PL, ts);
    const double* Ad = c.in(Ua, naux * n * PL, ta);
    const double* Bd = c.in(Ub, naux * n * PL, tb);
    double* T = c.inout(target, n * n * PL, tt);
    if (cplx) rr::diag_contract_kernel<2><<<rr::blocks_for(n * n), 256, 0, c.s>>>(T, Sd, Ad, Bd, n, naux);
    else rr::diag_contract_kernel<1><<<rr::blocks_for(n * n), 256, 0, c.s>>>(T, Sd, Ad, Bd, n, naux);
    RR_LAUNCH_CHECK();
    c.out(target, T, n * n * PL);
    c.finish(opts);
  });
}

int rr_sigma_accum_u(double* U, double alpha, int64_t n, int64_t naux, int32_t cplx, const double* D, const double* Wm,
                     const rr_opts* opts) {
  return sigma_api([&] {
    RR_REQUIRE(U && D && Wm && n >= 0 && naux >= 0, RR_ERR_ARG, "accumU: bad arguments");
    if (n == 0 || naux == 0) return;
    const int PL = cplx ? 2 : 1;
    rr::SigmaCtx c(opts);
    rr::DevBuf<double> td, tw, wc, tu;
    const double* Dd = c.in(D, naux * n * PL, td);
    const double* Wd = rr::real_operand(c.in(Wm, n * n, tw), n, cplx != 0, wc, c.s);
    double* Ud = c.inout(U, naux * n * PL, tu);
    rr::GemmDesc g;  // U += alpha D Wm^T
    g.cplx = cplx != 0;
    g.M = naux; g.N = n; g.K = n;
    g.A = Dd; g.lda = n; g.B = Wd; g.ldb = n; g.opB = rr::Op::T; g.C = Ud; g.ldc = n;
    g.alpha = alpha; g.beta = 1.0;
    rr::gemm(g, c.s);
    c.out(U, Ud, naux * n * PL);
    c.finish(opts);
  });
}

}  // extern "C"
