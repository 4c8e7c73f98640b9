// Test infrastructure only: a C-ABI bridge onto the reference's OWN RI functions, compiled
// unmodified from the reference source tree by oracle/Makefile into oracle/_ref/librrref.so.
// Only tests/, tests/golden/make_golden.py and bench.py's CPU-baseline leg load it; the product
// library never links it.  Every entry point copies plain row-major buffers into the reference's
// Matrix<T> value types, calls the reference function named in its comment, and copies the result
// back.  Complex buffers are interleaved (re, im) doubles, i.e. std::complex<double> layout.
// Errors (std::exception) are caught and reported as return code 1; 0 means success.
#include <omp.h>

#include <complex>
#include <cstdint>
#include <cstring>
#include <deque>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "C4_DHF.h"
#include "DIIS.h"
#include "LinearAlgebra.h"
#include "NonRelFockMatrixRi.h"
#include "NonRelHartreeFock.h"
#include "NonRelSpinRiMoEri.h"
#include "RiGemmFock.h"
#include "RiSigmaGemm.h"
#include "RiMoEri.h"
#include "UkbFockMatrixRi.h"
#include "X2C_FockMatrixRi.h"
#include "X2C_HF.h"
#include "JkOnlyFock.h"
#include "HartreeExchangeGradient.h"
#include "ADAM.h"
#include "HartreeExchangeHessian.h"
#include "OrbitalGradient.h"
#include "SpinorRotation.h"
#include "ThreeCenterIntegrals.h"
#include "RiSigmaHessianToolkit.h"
#include "Restart.h"
#include "CasFock.h"
#include "PnofFock.h"
#include "PNOFs.h"
#include "Tensor4.h"
#include "../include/rr_ri.h"

extern "C" void scipy_openblas_set_num_threads(int n);

using rerdmft::Matrix;
using C = std::complex<double>;
using i64 = std::int64_t;

namespace {

thread_local std::string g_last_error;

template <typename T>
Matrix<T> toMatrix(const T* p, i64 rows, i64 cols) {
  Matrix<T> m(static_cast<std::size_t>(rows), static_cast<std::size_t>(cols));
  if (rows * cols > 0) std::memcpy(m.data(), p, sizeof(T) * static_cast<std::size_t>(rows * cols));
  return m;
}
Matrix<C> toCMatrix(const double* p, i64 rows, i64 cols) {
  return toMatrix<C>(reinterpret_cast<const C*>(p), rows, cols);
}
template <typename T>
void fromMatrix(const Matrix<T>& m, T* out) {
  if (m.rows() * m.cols() > 0) std::memcpy(out, m.data(), sizeof(T) * m.rows() * m.cols());
}
void fromCMatrix(const Matrix<C>& m, double* out) { fromMatrix<C>(m, reinterpret_cast<C*>(out)); }

template <typename F>
int guard(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return 1;
  }
}

}  // namespace

// ---- Stubs for the non-RI overloads the SCF-loop translation units reference but the RI path
// never calls (their real definitions need libcint, which is absent).  Each one throws. ----
namespace rerdmft {
[[noreturn]] static void notBuilt(const char* what) {
  throw std::runtime_error(std::string(what) + ": non-RI two-electron path is not built into the oracle");
}
Matrix<double> nonRelFockMatrix(const Matrix<double>&, const AoCholesky&, const Matrix<double>&) {
  notBuilt("nonRelFockMatrix(AoCholesky)");
}
Matrix<C> x2cFockMatrix(const Matrix<C>&, const AoCholesky&, const Matrix<C>&) { notBuilt("x2cFockMatrix"); }
Matrix<C> x2cFockMatrix(const Matrix<C>&, const PackedTwoElectronTensor&, const Matrix<C>&) {
  notBuilt("x2cFockMatrix");
}
Matrix<C> x2cFockMatrix(const Matrix<C>&, const Tensor4<double>&, const Matrix<C>&) { notBuilt("x2cFockMatrix"); }
Matrix<C> rkbFockMatrix(const Matrix<C>&, const RkbCholesky&, const Matrix<C>&) { notBuilt("rkbFockMatrix"); }
Matrix<C> rkbFockMatrix(const Matrix<C>&, const SymmetricEri<C>&, const Matrix<C>&) { notBuilt("rkbFockMatrix"); }
Matrix<C> rkbFockMatrix(const Matrix<C>&, const UkbDirectEriSource&, const Matrix<C>&) {
  notBuilt("rkbFockMatrix");
}
template <>
double CholeskyEri<double>::operator()(std::size_t, std::size_t, std::size_t, std::size_t) const {
  notBuilt("CholeskyEri");
}
template <>
C CholeskyEri<C>::operator()(std::size_t, std::size_t, std::size_t, std::size_t) const { notBuilt("CholeskyEri"); }
}  // namespace rerdmft

extern "C" {

const char* rrref_last_error() { return g_last_error.c_str(); }

// OpenMP threads for the reference's parallel loops; BLAS stays serial inside them, exactly as
// the reference expects (src/Utils/BlasThreads.h).
void rrref_set_threads(int n) {
  scipy_openblas_set_num_threads(1);
  omp_set_num_threads(n > 0 ? n : 1);
}

// src/NON_REL/NonRelFockMatrixRi.cpp:71 nonRelFockMatrix(h, RiNonRelEriSource, D)
int rrref_nonrel_fock(i64 n, i64 naux, const double* B, const double* h, const double* D, const double* S,
                      const double* X, i64 n_eff, double* F) {
  return guard([&] {
    rerdmft::RiNonRelEriSource src;
    src.nl = static_cast<std::size_t>(n);
    src.eri3_L = toMatrix(B, naux, n * n);
    src.x_large = toMatrix(X, n, n_eff);
    src.overlap = toMatrix(S, n, n);
    fromMatrix(rerdmft::nonRelFockMatrix(toMatrix(h, n, n), src, toMatrix(D, n, n)), F);
  });
}

// src/X2C_DHF/X2C_FockMatrixRi.cpp:79 x2cFockMatrix(h_x2c, RiX2cEriSource, P); complex 2nl x 2nl.
int rrref_x2c_fock(i64 nl, i64 naux, const double* B, const double* h, const double* P, const double* S,
                   const double* X, i64 n_eff, double* F) {
  return guard([&] {
    rerdmft::RiX2cEriSource src;
    src.nl = static_cast<std::size_t>(nl);
    src.eri3_L = toMatrix(B, naux, nl * nl);
    src.x_large = toCMatrix(X, 2 * nl, n_eff);
    src.overlap = toCMatrix(S, 2 * nl, 2 * nl);
    fromCMatrix(rerdmft::x2cFockMatrix(toCMatrix(h, 2 * nl, 2 * nl), src, toCMatrix(P, 2 * nl, 2 * nl)), F);
  });
}

// src/UKB/UkbFockMatrixRi.cpp:35 riFockTwoElectronDirect(nl, ns, B_LL, B_SS, P_ukb, C_occ_ukb, occ)
int rrref_ukb_two_electron(i64 nl, i64 ns, i64 naux, const double* B_LL, const double* B_SS, const double* P_ukb,
                           const double* C_occ, i64 n_occ, const double* occ, double* G) {
  return guard([&] {
    const i64 nu = 2 * nl + 2 * ns;
    std::vector<double> o(occ, occ + n_occ);
    fromCMatrix(rerdmft::riFockTwoElectronDirect(static_cast<std::size_t>(nl), static_cast<std::size_t>(ns),
                                                 toMatrix(B_LL, naux, nl * nl), toMatrix(B_SS, naux, ns * ns),
                                                 toCMatrix(P_ukb, nu, nu), toCMatrix(C_occ, nu, n_occ), o),
                G);
  });
}

static rerdmft::RiDirectEriSource makeDirect(i64 nl, i64 ns, i64 naux, const double* B_LL, const double* B_SS,
                                             const double* v_total, i64 n_rkb, const double* s_full,
                                             const double* x_full, i64 n_eff) {
  rerdmft::RiDirectEriSource src;
  src.nl = static_cast<std::size_t>(nl);
  src.ns = static_cast<std::size_t>(ns);
  src.eri3_LL = toMatrix(B_LL, naux, nl * nl);
  src.eri3_SS = toMatrix(B_SS, naux, ns * ns);
  const i64 nu = 2 * nl + 2 * ns;
  if (v_total) src.v_total = toCMatrix(v_total, nu, n_rkb);
  if (s_full) src.s_full = toCMatrix(s_full, n_rkb, n_rkb);
  if (x_full) src.x_full = toCMatrix(x_full, n_rkb, n_eff);
  return src;
}

// src/UKB/UkbFockMatrixRi.cpp:185 rkbFockMatrix(h_rkb, RiDirectEriSource, P)
int rrref_rkb_fock(i64 nl, i64 ns, i64 naux, const double* B_LL, const double* B_SS, const double* v_total,
                   i64 n_rkb, const double* s_full, const double* x_full, i64 n_eff, const double* h,
                   const double* P, double* F) {
  return guard([&] {
    auto src = makeDirect(nl, ns, naux, B_LL, B_SS, v_total, n_rkb, s_full, x_full, n_eff);
    fromCMatrix(rerdmft::rkbFockMatrix(toCMatrix(h, n_rkb, n_rkb), src, toCMatrix(P, n_rkb, n_rkb)), F);
  });
}

// src/NON_REL/NonRelSpinRiMoEri.cpp:13 buildRiNonRelSpinMoEri(B, n, C)
int rrref_nonrel_mo_build(i64 n, i64 naux, const double* B, const double* Cs, double* out) {
  return guard([&] {
    auto eri = rerdmft::buildRiNonRelSpinMoEri(toMatrix(B, naux, n * n), static_cast<std::size_t>(n),
                                               toMatrix(Cs, n, n));
    fromMatrix(eri.b(), out);
  });
}

// src/NON_REL/NonRelSpinRiMoEri.cpp:45 RiNonRelSpinMoEri::rotated(U), U is 2n x 2n
int rrref_nonrel_mo_rotated(i64 n, i64 naux, const double* Bmo, const double* U, double* out) {
  return guard([&] {
    rerdmft::RiNonRelSpinMoEri eri(static_cast<std::size_t>(n), toMatrix(Bmo, naux, n * n));
    fromMatrix(eri.rotated(toMatrix(U, 2 * n, 2 * n)).b(), out);
  });
}

// src/NON_REL/NonRelSpinRiMoEri.h:77 embeddedB()
int rrref_nonrel_mo_embedded(i64 n, i64 naux, const double* Bmo, double* out) {
  return guard([&] {
    rerdmft::RiNonRelSpinMoEri eri(static_cast<std::size_t>(n), toMatrix(Bmo, naux, n * n));
    fromMatrix(eri.embeddedB(), out);
  });
}

// src/NON_REL/NonRelSpinRiMoEri.h:40 operator()(a,b,c,d) over `count` index quadruples.
int rrref_nonrel_mo_eri(i64 n, i64 naux, const double* Bmo, i64 count, const i64* abcd, double* out) {
  return guard([&] {
    rerdmft::RiNonRelSpinMoEri eri(static_cast<std::size_t>(n), toMatrix(Bmo, naux, n * n));
    for (i64 t = 0; t < count; ++t)
      out[t] = eri(static_cast<std::size_t>(abcd[4 * t]), static_cast<std::size_t>(abcd[4 * t + 1]),
                   static_cast<std::size_t>(abcd[4 * t + 2]), static_cast<std::size_t>(abcd[4 * t + 3]));
  });
}

// src/UKB/RiMoEri.cpp:64 buildRiMoEri(RiDirectEriSource, c_ukb); c_ukb is n_ukb x n_total complex.
int rrref_ri_mo_build(i64 nl, i64 ns, i64 naux, const double* B_LL, const double* B_SS, const double* c_ukb,
                      i64 n_total, double* out) {
  return guard([&] {
    auto src = makeDirect(nl, ns, naux, B_LL, B_SS, nullptr, 0, nullptr, nullptr, 0);
    fromCMatrix(rerdmft::buildRiMoEri(src, toCMatrix(c_ukb, 2 * nl + 2 * ns, n_total)).b(), out);
  });
}

// src/UKB/RiMoEri.cpp:88 RiMoEri::rotated(U)
int rrref_ri_mo_rotated(i64 n, i64 naux, const double* Bmo, const double* U, double* out) {
  return guard([&] {
    rerdmft::RiMoEri eri(static_cast<std::size_t>(n), toCMatrix(Bmo, naux, n * n));
    fromCMatrix(eri.rotated(toCMatrix(U, n, n)).b(), out);
  });
}

// src/UKB/RiMoEri.cpp:112 RiMoEri::positiveBlock(off)
int rrref_ri_mo_positive(i64 n, i64 naux, const double* Bmo, i64 off, double* out) {
  return guard([&] {
    rerdmft::RiMoEri eri(static_cast<std::size_t>(n), toCMatrix(Bmo, naux, n * n));
    fromCMatrix(eri.positiveBlock(static_cast<std::size_t>(off)).b(), out);
  });
}

// src/UKB/RiMoEri.h:50 operator()(a,b,c,d) over `count` quadruples; out is complex.
int rrref_ri_mo_eri(i64 n, i64 naux, const double* Bmo, i64 count, const i64* abcd, double* out) {
  return guard([&] {
    rerdmft::RiMoEri eri(static_cast<std::size_t>(n), toCMatrix(Bmo, naux, n * n));
    C* o = reinterpret_cast<C*>(out);
    for (i64 t = 0; t < count; ++t)
      o[t] = eri(static_cast<std::size_t>(abcd[4 * t]), static_cast<std::size_t>(abcd[4 * t + 1]),
                 static_cast<std::size_t>(abcd[4 * t + 2]), static_cast<std::size_t>(abcd[4 * t + 3]));
  });
}

static std::vector<std::size_t> pairVec(const i64* pair_of, i64 n) {
  std::vector<std::size_t> v;
  if (pair_of)
    for (i64 i = 0; i < n; ++i) v.push_back(static_cast<std::size_t>(pair_of[i]));
  return v;
}

// src/Hessian_opt/RiGemmFock.cpp:173 hartreeExchangeFockMatrix(h, RiNonRelSpinMoEri, ...): n_sp spatial
// orbitals, h/h2/x2/l1/l2 are (2 n_sp)^2; pair_of may be null (no L terms).  use_reference selects the
// reference's own element-by-element A/B path (RERDMFT_RI_HV_REFERENCE).
int rrref_hx_fock_nonrel(i64 n_sp, i64 naux, const double* Bmo, const double* h, const double* occ,
                         const double* h2, const double* x2, const i64* pair_of, const double* l1,
                         const double* l2, int use_reference, double* F) {
  return guard([&] {
    const i64 n = 2 * n_sp;
    rerdmft::risigma::useReferenceFlag() = use_reference != 0;
    rerdmft::RiNonRelSpinMoEri eri(static_cast<std::size_t>(n_sp), toMatrix(Bmo, naux, n_sp * n_sp));
    std::vector<double> o(occ, occ + n);
    Matrix<double> L1 = pair_of ? toMatrix(l1, n, n) : Matrix<double>();
    Matrix<double> L2 = pair_of ? toMatrix(l2, n, n) : Matrix<double>();
    auto f = rerdmft::hartreeExchangeFockMatrix(toMatrix(h, n, n), eri, o, toMatrix(h2, n, n), toMatrix(x2, n, n),
                                                pairVec(pair_of, n), L1, L2);
    rerdmft::risigma::useReferenceFlag() = false;
    fromMatrix(f, F);
  });
}

// src/Hessian_opt/RiGemmFock.cpp:161 hartreeExchangeFockMatrix(h, RiMoEri, ...): complex, n x n.
int rrref_hx_fock_complex(i64 n, i64 naux, const double* Bmo, const double* h, const double* occ, const double* h2,
                          const double* x2, const i64* pair_of, const double* l1, const double* l2,
                          int use_reference, double* F) {
  return guard([&] {
    rerdmft::risigma::useReferenceFlag() = use_reference != 0;
    rerdmft::RiMoEri eri(static_cast<std::size_t>(n), toCMatrix(Bmo, naux, n * n));
    std::vector<double> o(occ, occ + n);
    Matrix<double> L1 = pair_of ? toMatrix(l1, n, n) : Matrix<double>();
    Matrix<double> L2 = pair_of ? toMatrix(l2, n, n) : Matrix<double>();
    auto f = rerdmft::hartreeExchangeFockMatrix(toCMatrix(h, n, n), eri, o, toMatrix(h2, n, n), toMatrix(x2, n, n),
                                                pairVec(pair_of, n), L1, L2);
    rerdmft::risigma::useReferenceFlag() = false;
    fromCMatrix(f, F);
  });
}

// src/Utils/DIIS.cpp:53 scfCommutatorError (real and complex)
int rrref_commutator_error_real(i64 n, const double* F, const double* P, const double* S, double* E) {
  return guard([&] {
    fromMatrix(rerdmft::scfCommutatorError(toMatrix(F, n, n), toMatrix(P, n, n), toMatrix(S, n, n)), E);
  });
}
int rrref_commutator_error_complex(i64 n, const double* F, const double* P, const double* S, double* E) {
  return guard([&] {
    fromCMatrix(rerdmft::scfCommutatorError(toCMatrix(F, n, n), toCMatrix(P, n, n), toCMatrix(S, n, n)), E);
  });
}

// src/Utils/DIIS.cpp:79 Diis<T>::extrapolate, driven over a whole sequence: step t feeds
// (errors[t], values[t]) into one Diis object and writes its result to out[t]; weights_count[t]
// receives lastWeights().size().  is_complex selects Diis<complex<double>>.
int rrref_diis_sequence(int is_complex, i64 max_vectors, i64 steps, i64 size, const double* errors,
                        const double* values, double* out, i64* weights_count) {
  return guard([&] {
    const i64 stride = is_complex ? 2 * size : size;
    if (is_complex) {
      rerdmft::Diis<C> d(static_cast<std::size_t>(max_vectors));
      for (i64 t = 0; t < steps; ++t) {
        auto r = d.extrapolate(toCMatrix(errors + t * stride, 1, size), toCMatrix(values + t * stride, 1, size));
        fromCMatrix(r, out + t * stride);
        weights_count[t] = static_cast<i64>(d.lastWeights().size());
      }
    } else {
      rerdmft::Diis<double> d(static_cast<std::size_t>(max_vectors));
      for (i64 t = 0; t < steps; ++t) {
        auto r = d.extrapolate(toMatrix(errors + t * stride, 1, size), toMatrix(values + t * stride, 1, size));
        fromMatrix(r, out + t * stride);
        weights_count[t] = static_cast<i64>(d.lastWeights().size());
      }
    }
  });
}

// src/Linear_Algebra/LinearAlgebra.cpp:267 canonicalOrthogonalize; X_out must hold n*n doubles.
int rrref_canonical_orth(i64 n, const double* S, double thr, double* X_out, i64* n_eff) {
  return guard([&] {
    auto x = rerdmft::canonicalOrthogonalize(toMatrix(S, n, n), thr);
    *n_eff = static_cast<i64>(x.cols());
    fromMatrix(x, X_out);
  });
}
// canonicalOrthogonalize / canonicalOrthogonalizeHermitian with the RankReductionReport
// (src/Linear_Algebra/LinearAlgebra.cpp:267 and :312): report = {n_kept, n_dropped, smallest_kept,
// largest_dropped}.
int rrref_canonical_orth_report(i64 n, const double* S, int hermitian, double thr, double* X_out, i64* n_eff,
                                double* report) {
  return guard([&] {
    rerdmft::RankReductionReport r;
    if (hermitian) {
      auto x = rerdmft::canonicalOrthogonalizeHermitian(toCMatrix(S, n, n), thr, &r);
      *n_eff = static_cast<i64>(x.cols());
      fromCMatrix(x, X_out);
    } else {
      auto x = rerdmft::canonicalOrthogonalize(toMatrix(S, n, n), thr, &r);
      *n_eff = static_cast<i64>(x.cols());
      fromMatrix(x, X_out);
    }
    report[0] = static_cast<double>(r.n_kept);
    report[1] = static_cast<double>(r.n_dropped);
    report[2] = r.smallest_kept;
    report[3] = r.largest_dropped;
  });
}
}  // extern "C": the helpers below are templates

// ---- RI sigma-vector Hessian-vector primitives (src/Hessian_opt/RiSigmaGemm.cpp,
// src/Hessian_opt/RiSigmaHessianToolkit.cpp).  Complex operands are interleaved (cplx = 1).

template <typename T>
static rerdmft::Matrix<T> sigmaMat(const double* p, i64 r, i64 c) {
  if constexpr (std::is_same_v<T, double>) return toMatrix(p, r, c);
  else return toCMatrix(p, r, c);
}
template <typename T>
static void sigmaOut(const rerdmft::Matrix<T>& m, double* out) {
  if constexpr (std::is_same_v<T, double>) fromMatrix(m, out);
  else fromCMatrix(m, out);
}
template <typename T>
static void sigmaVecOut(const std::vector<T>& v, double* out) {
  std::memcpy(out, v.data(), sizeof(T) * v.size());
}

template <typename T>
static void sigmaToolkit(i64 n, i64 naux, const double* B, const double* K, double* kb1, double* kb2, double* bdiag,
                         double* kb1diag, double* kb2diag) {
  auto b = sigmaMat<T>(B, naux, n * n);
  auto t = rerdmft::buildRiSigmaHessianToolkit<T>(static_cast<std::size_t>(n), b, toMatrix(K, n, n));
  sigmaOut(t.kb1, kb1);
  sigmaOut(t.kb2, kb2);
  sigmaVecOut(t.bdiag, bdiag);
  sigmaVecOut(t.kb1diag, kb1diag);
  sigmaVecOut(t.kb2diag, kb2diag);
}

// One PairOp from flat tables: s (naux x n^2, nullable), idx (n^2 uint32), w (n^2, nullable), row
// (naux x n, nullable), post (real n x n, nullable).
template <typename T>
struct SigmaOp {
  rerdmft::Matrix<T> s, row;
  rerdmft::Matrix<double> post;
  rerdmft::risigma::PairOp<T> op;
  SigmaOp(i64 n, i64 naux, const double* sp, const std::uint32_t* idx, const double* w, const double* rowp,
          const double* postp) {
    const std::size_t n2 = static_cast<std::size_t>(n * n);
    if (sp) {
      s = sigmaMat<T>(sp, naux, n * n);
      op.s = &s;
      op.idx.assign(idx, idx + n2);
    }
    if (w) op.w.assign(w, w + n2);
    if (rowp) {
      row = sigmaMat<T>(rowp, naux, n);
      op.row = &row;
    }
    if (postp) {
      post = toMatrix(postp, n, n);
      op.post = &post;
    }
  }
};

template <typename T>
static void sigmaPair(i64 n, i64 naux, double sign, double* target, const double* fs, const std::uint32_t* fidx,
                      const double* fw, const double* frow, const double* fpost, const double* gs,
                      const std::uint32_t* gidx, const double* gw, const double* grow, const double* gpost) {
  auto tgt = sigmaMat<T>(target, n, n);
  SigmaOp<T> f(n, naux, fs, fidx, fw, frow, fpost), g(n, naux, gs, gidx, gw, grow, gpost);
  rerdmft::risigma::pairContract<T>(tgt, sign, static_cast<std::size_t>(n), static_cast<std::size_t>(naux), f.op,
                                    g.op);
  sigmaOut(tgt, target);
}

template <typename T>
static void sigmaDiag(i64 n, i64 naux, double* target, const double* S, const double* Ua, const double* Ub) {
  auto tgt = sigmaMat<T>(target, n, n);
  auto s = sigmaMat<T>(S, naux, n * n);
  rerdmft::Matrix<T> ua, ub;
  if (Ua) ua = sigmaMat<T>(Ua, naux, n);
  if (Ub) ub = sigmaMat<T>(Ub, naux, n);
  rerdmft::risigma::diagContract<T>(tgt, static_cast<std::size_t>(n), static_cast<std::size_t>(naux), s,
                                    Ua ? &ua : nullptr, Ub ? &ub : nullptr);
  sigmaOut(tgt, target);
}

template <typename T>
static void sigmaAccum(i64 n, i64 naux, double* U, double alpha, const double* D, const double* Wm) {
  auto u = sigmaMat<T>(U, naux, n);
  std::vector<T> d(static_cast<std::size_t>(naux * n));
  std::memcpy(d.data(), D, sizeof(T) * d.size());
  rerdmft::risigma::accumU<T>(u, alpha, static_cast<std::size_t>(n), static_cast<std::size_t>(naux), d,
                              toMatrix(Wm, n, n));
  sigmaOut(u, U);
}

extern "C" {

int rrref_sigma_toolkit(i64 n, i64 naux, int cplx, const double* B, const double* K, double* kb1, double* kb2,
                        double* bdiag, double* kb1diag, double* kb2diag) {
  return guard([&] {
    if (cplx) sigmaToolkit<std::complex<double>>(n, naux, B, K, kb1, kb2, bdiag, kb1diag, kb2diag);
    else sigmaToolkit<double>(n, naux, B, K, kb1, kb2, bdiag, kb1diag, kb2diag);
  });
}

int rrref_sigma_pair_contract(i64 n, i64 naux, int cplx, double sign, double* target, const double* fs,
                              const std::uint32_t* fidx, const double* fw, const double* frow, const double* fpost,
                              const double* gs, const std::uint32_t* gidx, const double* gw, const double* grow,
                              const double* gpost) {
  return guard([&] {
    if (cplx)
      sigmaPair<std::complex<double>>(n, naux, sign, target, fs, fidx, fw, frow, fpost, gs, gidx, gw, grow, gpost);
    else
      sigmaPair<double>(n, naux, sign, target, fs, fidx, fw, frow, fpost, gs, gidx, gw, grow, gpost);
  });
}

int rrref_sigma_diag_contract(i64 n, i64 naux, int cplx, double* target, const double* S, const double* Ua,
                              const double* Ub) {
  return guard([&] {
    if (cplx) sigmaDiag<std::complex<double>>(n, naux, target, S, Ua, Ub);
    else sigmaDiag<double>(n, naux, target, S, Ua, Ub);
  });
}

int rrref_sigma_accum_u(i64 n, i64 naux, int cplx, double* U, double alpha, const double* D, const double* Wm) {
  return guard([&] {
    if (cplx) sigmaAccum<std::complex<double>>(n, naux, U, alpha, D, Wm);
    else sigmaAccum<double>(n, naux, U, alpha, D, Wm);
  });
}

// src/Hessian_opt/HartreeExchangeHessian.cpp:653 hartreeExchangeJointHessianDiagonal, RiMoEri instantiation
// (:705-711): out (2 npairs); pairs npairs x 2; pair_of null = no pair terms.
int rrref_hx_joint_hessian_diag(i64 n, i64 naux, const double* Bmo, const double* h, const double* occ,
                                const double* h2, const double* x2, const double* fock, i64 npairs, const i64* pairs,
                                const i64* pair_of, const double* l1, const double* l2, double* out) {
  return guard([&] {
    rerdmft::RiMoEri eri(static_cast<std::size_t>(n), toCMatrix(Bmo, naux, n * n));
    std::vector<std::pair<std::size_t, std::size_t>> pr(static_cast<std::size_t>(npairs));
    for (i64 i = 0; i < npairs; ++i) pr[i] = {static_cast<std::size_t>(pairs[2 * i]), static_cast<std::size_t>(pairs[2 * i + 1])};
    std::vector<std::size_t> po;
    rerdmft::Matrix<double> L1, L2;
    if (pair_of) {
      po.assign(pair_of, pair_of + n);
      L1 = toMatrix(l1, n, n);
      L2 = toMatrix(l2, n, n);
    }
    auto d = rerdmft::hartreeExchangeJointHessianDiagonal(toCMatrix(h, n, n), eri, std::vector<double>(occ, occ + n),
                                                          toMatrix(h2, n, n), toMatrix(x2, n, n), toCMatrix(fock, n, n),
                                                          pr, po, L1, L2);
    std::memcpy(out, d.data(), sizeof(double) * d.size());
  });
}

// src/Hessian_opt/PnofFock.cpp:29 buildPnofFullTwoRdm and :139 buildPnofPairOf: functional 0..3 = PNOF5,
// PNOF7, PNOF7s, GNOF; geminals n_gem x 4 (i, ibar, subspace_id, is_principal).
int rrref_pnof_full_two_rdm(int functional, i64 n_gem, const i64* gem, const double* occ, i64 n_total,
                            int relativistic, double* h2, double* x2, double* l1, double* l2, i64* pair_of) {
  return guard([&] {
    std::vector<rerdmft::PnofGeminal> g(static_cast<std::size_t>(n_gem));
    for (i64 k = 0; k < n_gem; ++k)
      g[k] = rerdmft::PnofGeminal{static_cast<std::size_t>(gem[4 * k]), static_cast<std::size_t>(gem[4 * k + 1]),
                                  static_cast<std::size_t>(gem[4 * k + 2]), gem[4 * k + 3] != 0};
    const rerdmft::PnofFunctional f = functional == 0 ? rerdmft::PnofFunctional::kPnof5
                                      : functional == 1 ? rerdmft::PnofFunctional::kPnof7
                                      : functional == 2 ? rerdmft::PnofFunctional::kPnof7s
                                                        : rerdmft::PnofFunctional::kGnof;
    auto full = rerdmft::buildPnofFullTwoRdm(f, g, std::vector<double>(occ, occ + n_total),
                                             static_cast<std::size_t>(n_total), relativistic != 0);
    fromMatrix(full.two_rdm_h, h2);
    fromMatrix(full.two_rdm_x, x2);
    fromMatrix(full.two_rdm_l1, l1);
    fromMatrix(full.two_rdm_l2, l2);
    auto po = rerdmft::buildPnofPairOf(g, static_cast<std::size_t>(n_total));
    for (i64 i = 0; i < n_total; ++i) pair_of[i] = static_cast<i64>(po[i]);
  });
}

// src/Occ_opt/PNOFs.cpp:271 pnofElectronicEnergy (with :212 buildPnofTwoRdm) and :463
// pnofOccupationGradient for a non-relativistic spin-orbital problem: the RiNonRelSpinMoEri of Bmo (n_sp
// spatial orbitals) expanded to the dense Tensor4<double> over its 2 n_sp accessors (the instantiations the
// reference compiles), h 2n x 2n, occupations 2n; geminals n_gem x 4 as for rrref_pnof_full_two_rdm.
int rrref_pnof_energy_nonrel(int functional, i64 n_gem, const i64* gem, const double* occ, i64 n_sp, i64 naux,
                             const double* Bmo, const double* h, double* energy, double* grad) {
  return guard([&] {
    std::vector<rerdmft::PnofGeminal> g(static_cast<std::size_t>(n_gem));
    for (i64 k = 0; k < n_gem; ++k)
      g[k] = rerdmft::PnofGeminal{static_cast<std::size_t>(gem[4 * k]), static_cast<std::size_t>(gem[4 * k + 1]),
                                  static_cast<std::size_t>(gem[4 * k + 2]), gem[4 * k + 3] != 0};
    const rerdmft::PnofFunctional f = functional == 0 ? rerdmft::PnofFunctional::kPnof5
                                      : functional == 1 ? rerdmft::PnofFunctional::kPnof7
                                      : functional == 2 ? rerdmft::PnofFunctional::kPnof7s
                                                        : rerdmft::PnofFunctional::kGnof;
    rerdmft::RiNonRelSpinMoEri eri(static_cast<std::size_t>(n_sp), toMatrix(Bmo, naux, n_sp * n_sp));
    const std::size_t d = static_cast<std::size_t>(2 * n_sp);
    rerdmft::Tensor4<double> t(d, d, d, d);
    for (std::size_t a = 0; a < d; ++a)
      for (std::size_t b = 0; b < d; ++b)
        for (std::size_t c = 0; c < d; ++c)
          for (std::size_t e = 0; e < d; ++e) t(a, b, c, e) = eri(a, b, c, e);
    const std::vector<double> o(occ, occ + d);
    const auto H = toMatrix(h, static_cast<i64>(d), static_cast<i64>(d));
    const auto two = rerdmft::buildPnofTwoRdm(f, g, o, false);
    *energy = rerdmft::pnofElectronicEnergy(f, H, t, o, g, two, false);
    if (grad) {
      const auto gr = rerdmft::pnofOccupationGradient(f, H, t, o, g, false);
      std::memcpy(grad, gr.data(), sizeof(double) * gr.size());
    }
  });
}

// The CASSCF RI overloads (src/MCSCF/CasFock.cpp:246-262) on an MO tensor: kind 0 = RiNonRelSpinMoEri
// (real spatial tensor of n orbitals, accessor dimension 2n), 1 = RiMoEri (complex, n spinors).
// casTwoElectronOperator: G (d x d) from rho (d x d).
int rrref_cas_two_electron(int kind, i64 n, i64 naux, const double* Bmo, const double* rho, double* G) {
  return guard([&] {
    if (kind == 0) {
      rerdmft::RiNonRelSpinMoEri eri(static_cast<std::size_t>(n), toMatrix(Bmo, naux, n * n));
      fromMatrix(rerdmft::casTwoElectronOperator(eri, toMatrix(rho, 2 * n, 2 * n)), G);
    } else {
      rerdmft::RiMoEri eri(static_cast<std::size_t>(n), toCMatrix(Bmo, naux, n * n));
      fromCMatrix(rerdmft::casTwoElectronOperator(eri, toCMatrix(rho, n, n)), G);
    }
  });
}
// casActiveCumulantFock: F (d x a) from the active list and lambda (a^4, [s,t,r,q]).
int rrref_cas_cumulant_fock(int kind, i64 n, i64 naux, const double* Bmo, i64 a, const i64* active,
                            const double* lambda, double* F) {
  return guard([&] {
    std::vector<std::size_t> act(active, active + a);
    const std::size_t a4 = static_cast<std::size_t>(a * a * a * a);
    if (kind == 0) {
      rerdmft::RiNonRelSpinMoEri eri(static_cast<std::size_t>(n), toMatrix(Bmo, naux, n * n));
      fromMatrix(rerdmft::casActiveCumulantFock(eri, act, std::vector<double>(lambda, lambda + a4)), F);
    } else {
      rerdmft::RiMoEri eri(static_cast<std::size_t>(n), toCMatrix(Bmo, naux, n * n));
      const auto* lc = reinterpret_cast<const std::complex<double>*>(lambda);
      fromCMatrix(rerdmft::casActiveCumulantFock(eri, act, std::vector<std::complex<double>>(lc, lc + a4)), F);
    }
  });
}
// casActiveIntegrals: (tu|vw) over the active list, a^4 values.
int rrref_cas_active_integrals(int kind, i64 n, i64 naux, const double* Bmo, i64 a, const i64* active, double* out) {
  return guard([&] {
    std::vector<std::size_t> act(active, active + a);
    if (kind == 0) {
      rerdmft::RiNonRelSpinMoEri eri(static_cast<std::size_t>(n), toMatrix(Bmo, naux, n * n));
      auto v = rerdmft::casActiveIntegrals(eri, act);
      std::memcpy(out, v.data(), sizeof(double) * v.size());
    } else {
      rerdmft::RiMoEri eri(static_cast<std::size_t>(n), toCMatrix(Bmo, naux, n * n));
      auto v = rerdmft::casActiveIntegrals(eri, act);
      std::memcpy(out, v.data(), sizeof(std::complex<double>) * v.size());
    }
  });
}

// src/Utils/Restart.cpp:94 writeRestart from the fields of an rr_restart record (the library's C
// struct, used here only as a carrier of the same fields).
int rrref_restart_write(const char* path, const rr_restart* r) {
  return guard([&] {
    rerdmft::RestartData d;
    d.method = r->method ? r->method : "";
    d.functional = r->functional ? r->functional : "";
    d.kind = r->kind ? r->kind : "";
    d.basis_fingerprint = r->basis_fingerprint;
    d.n_electrons = r->n_electrons;
    d.pnof_subspaces = r->pnof_subspaces;
    d.pnof_coupling = r->pnof_coupling;
    d.n_core = r->n_core;
    d.jk_frozen_pairs = r->jk_frozen_pairs;
    d.jk_active_pairs = r->jk_active_pairs;
    d.total_energy = r->total_energy;
    d.orbitals_optimized = r->orbitals_optimized != 0;
    d.converged = r->converged != 0;
    auto vec = [](const double* p, i64 n) { return p && n > 0 ? std::vector<double>(p, p + n) : std::vector<double>(); };
    d.occupations = vec(r->occupations, r->n_occupations);
    d.gammas = vec(r->gammas, r->n_gammas);
    d.amplitudes = vec(r->amplitudes, r->n_amplitudes);
    d.complex_coefficients = r->complex_coefficients != 0;
    d.rows = static_cast<std::uint64_t>(r->rows);
    d.cols = static_cast<std::uint64_t>(r->cols);
    d.coefficients = vec(r->coefficients, r->rows * r->cols * (r->complex_coefficients ? 2 : 1));
    d.cas_electrons = r->cas_electrons;
    d.cas_spinors = r->cas_spinors;
    d.cas_state = vec(r->cas_state, r->n_cas_state);
    rerdmft::writeRestart(path, d);
  });
}

// src/Utils/Restart.cpp:147 readRestart then :94 writeRestart: in_path parsed by the reference's reader
// and written back by its writer (a byte-identical out_path shows the reader took every field).
int rrref_restart_rewrite(const char* in_path, const char* out_path) {
  return guard([&] { rerdmft::writeRestart(out_path, rerdmft::readRestart(in_path)); });
}

// src/AO_ints/ThreeCenterIntegrals.cpp:191 transformRiThreeCenterAoLegs: out (naux, n_out^2) =
// t^T B^P t per aux row, t is n_ao x n_out.
int rrref_transform_ao_legs(i64 naux, i64 n_ao, const double* B, i64 n_out, const double* t, double* out) {
  return guard([&] {
    auto r = rerdmft::transformRiThreeCenterAoLegs(toMatrix(B, naux, n_ao * n_ao), static_cast<std::size_t>(n_ao),
                                                   toMatrix(t, n_ao, n_out));
    fromMatrix(r, out);
  });
}
// src/Linear_Algebra/LinearAlgebra.cpp:312 canonicalOrthogonalizeHermitian; X_out holds n*n complex.
int rrref_canonical_orth_hermitian(i64 n, const double* S, double thr, double* X_out, i64* n_eff) {
  return guard([&] {
    auto x = rerdmft::canonicalOrthogonalizeHermitian(toCMatrix(S, n, n), thr);
    *n_eff = static_cast<i64>(x.cols());
    fromCMatrix(x, X_out);
  });
}
// src/Linear_Algebra/LinearAlgebra.cpp:51 / :122 diagonalizeSymmetric / diagonalizeHermitian
int rrref_diag_sym(i64 n, const double* A, double* w, double* V) {
  return guard([&] {
    auto r = rerdmft::diagonalizeSymmetric(toMatrix(A, n, n));
    std::memcpy(w, r.eigenvalues.data(), sizeof(double) * static_cast<std::size_t>(n));
    fromMatrix(r.eigenvectors, V);
  });
}
int rrref_diag_herm(i64 n, const double* A, double* w, double* V) {
  return guard([&] {
    auto r = rerdmft::diagonalizeHermitian(toCMatrix(A, n, n));
    std::memcpy(w, r.eigenvalues.data(), sizeof(double) * static_cast<std::size_t>(n));
    fromCMatrix(r.eigenvectors, V);
  });
}

// SCF result record shared by the three loop wrappers below.
struct rrref_scf_result {
  double electronic_energy;
  i64 iterations;
  i64 converged;
};

static void copyHistory(const std::vector<double>& e, double* hist, i64 max_iter) {
  for (std::size_t i = 0; i < e.size() && static_cast<i64>(i) < max_iter; ++i) hist[i] = e[i];
}

// The result's orbital_energies, coefficients and Fock matrix, into the optional (nullable) outputs.
static void copyOrbitalsReal(const std::vector<double>& w, const rerdmft::Matrix<double>& c,
                             const rerdmft::Matrix<double>& f, double* w_out, double* c_out, double* f_out) {
  if (w_out) std::memcpy(w_out, w.data(), sizeof(double) * w.size());
  if (c_out) fromMatrix(c, c_out);
  if (f_out) fromMatrix(f, f_out);
}
static void copyOrbitalsComplex(const std::vector<double>& w, const rerdmft::Matrix<std::complex<double>>& c,
                                const rerdmft::Matrix<std::complex<double>>& f, double* w_out, double* c_out,
                                double* f_out) {
  if (w_out) std::memcpy(w_out, w.data(), sizeof(double) * w.size());
  if (c_out) fromCMatrix(c, c_out);
  if (f_out) fromCMatrix(f, f_out);
}

// src/NON_REL/NonRelHartreeFock.cpp:219 runNonRelativisticHartreeFock(RiNonRelEriSource, ...) with an
// empty geometry (nuclear repulsion 0).  energy_history gets one electronic energy per iteration.
int rrref_nonrel_scf(i64 n, i64 naux, const double* B, const double* h, const double* X, i64 n_eff,
                     const double* S, const double* P0, int n_electrons, int diis_size, int max_iter, double e_tol,
                     double d_tol, rrref_scf_result* res, double* P_out, double* energy_history, double* w_out,
                     double* c_out, double* f_out) {
  return guard([&] {
    rerdmft::RiNonRelEriSource src;
    src.nl = static_cast<std::size_t>(n);
    src.eri3_L = toMatrix(B, naux, n * n);
    src.x_large = toMatrix(X, n, n_eff);
    src.overlap = toMatrix(S, n, n);
    auto r = rerdmft::runNonRelativisticHartreeFock(src, toMatrix(h, n, n), src.x_large, toMatrix(P0, n, n),
                                                     n_electrons, {}, 1.0, src.overlap, diis_size, max_iter, e_tol,
                                                     d_tol);
    res->electronic_energy = r.electronic_energy;
    res->iterations = r.iterations;
    res->converged = r.converged ? 1 : 0;
    fromMatrix(r.density_matrix, P_out);
    copyOrbitalsReal(r.orbital_energies, r.c_matrix, r.fock_matrix, w_out, c_out, f_out);
    std::vector<double> e;
    for (const auto& rec : r.history) e.push_back(rec.energy);
    copyHistory(e, energy_history, max_iter);
  });
}

// src/X2C_DHF/X2C_HF.cpp:175 runX2CHartreeFockScf(h_x2c, RiX2cEriSource, ...)
int rrref_x2c_scf(i64 nl, i64 naux, const double* B, const double* h, const double* X, i64 n_eff, const double* S,
                  const double* P0, int n_electrons, int diis_size, int max_iter, double e_tol, double d_tol,
                  int kramers, rrref_scf_result* res, double* P_out, double* energy_history, double* w_out,
                  double* c_out, double* f_out) {
  return guard([&] {
    rerdmft::RiX2cEriSource src;
    src.nl = static_cast<std::size_t>(nl);
    src.eri3_L = toMatrix(B, naux, nl * nl);
    src.x_large = toCMatrix(X, 2 * nl, n_eff);
    src.overlap = toCMatrix(S, 2 * nl, 2 * nl);
    auto r = rerdmft::runX2CHartreeFockScf(toCMatrix(h, 2 * nl, 2 * nl), src, src.x_large,
                                           toCMatrix(P0, 2 * nl, 2 * nl), n_electrons, {}, 1.0, src.overlap,
                                           diis_size, max_iter, e_tol, d_tol, kramers != 0);
    res->electronic_energy = r.electronic_energy;
    res->iterations = r.iterations;
    res->converged = r.converged ? 1 : 0;
    fromCMatrix(r.density_matrix, P_out);
    copyOrbitalsComplex(r.orbital_energies, r.c_matrix, r.fock_matrix, w_out, c_out, f_out);
    std::vector<double> e;
    for (const auto& rec : r.history) e.push_back(rec.energy);
    copyHistory(e, energy_history, max_iter);
  });
}

// src/C4_DHF/C4_DHF.cpp:178 runDiracHartreeFockScf(h_rkb, RiDirectEriSource, ...)
int rrref_dhf_scf(i64 nl, i64 ns, i64 naux, const double* B_LL, const double* B_SS, const double* v_total,
                  i64 n_rkb, const double* s_full, const double* x_full, i64 n_eff, const double* h,
                  const double* P0, int n_electrons, int diis_size, int max_iter, double e_tol, double d_tol,
                  int kramers, rrref_scf_result* res, double* P_out, double* energy_history, double* w_out,
                  double* c_out, double* f_out) {
  return guard([&] {
    auto src = makeDirect(nl, ns, naux, B_LL, B_SS, v_total, n_rkb, s_full, x_full, n_eff);
    auto r = rerdmft::runDiracHartreeFockScf(toCMatrix(h, n_rkb, n_rkb), src, src.x_full,
                                             toCMatrix(P0, n_rkb, n_rkb), n_electrons, {}, 1.0, src.s_full,
                                             diis_size, max_iter, e_tol, d_tol, kramers != 0);
    res->electronic_energy = r.electronic_energy;
    res->iterations = r.iterations;
    res->converged = r.converged ? 1 : 0;
    fromCMatrix(r.density_matrix, P_out);
    copyOrbitalsComplex(r.orbital_energies, r.c_dhf, r.fock_matrix, w_out, c_out, f_out);
    std::vector<double> e;
    for (const auto& rec : r.history) e.push_back(rec.energy);
    copyHistory(e, energy_history, max_iter);
  });
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Orbital-rotation optimisation (functional stage): ADAM, rotations, gradient, Hessian diagonal.

namespace {

rerdmft::AdamOptions adamOptions(double lr, double b1, double b2, double eps) {
  rerdmft::AdamOptions o;
  o.learning_rate = lr;
  o.beta1 = b1;
  o.beta2 = b2;
  o.epsilon = eps;
  return o;
}

// E(x) = sum_i (a_i x_i^2 / 2 + b_i x_i) + c (sum_i x_i^2)^2, x += step: a deterministic
// AdamProblem for checking the run / restart logic.
class QuadraticProblem : public rerdmft::AdamProblem<double> {
 public:
  QuadraticProblem(std::vector<double> a, std::vector<double> b, double c, std::vector<double> x)
      : a_(std::move(a)), b_(std::move(b)), c_(c), x_(std::move(x)), best_(x_) {}
  std::size_t dimension() const override { return x_.size(); }
  double energy() override {
    double e = 0.0, r = 0.0;
    for (std::size_t i = 0; i < x_.size(); ++i) {
      e += 0.5 * a_[i] * x_[i] * x_[i] + b_[i] * x_[i];
      r += x_[i] * x_[i];
    }
    return e + c_ * r * r;
  }
  std::vector<double> gradient() override {
    double r = 0.0;
    for (double v : x_) r += v * v;
    std::vector<double> g(x_.size());
    for (std::size_t i = 0; i < x_.size(); ++i) g[i] = a_[i] * x_[i] + b_[i] + 4.0 * c_ * r * x_[i];
    return g;
  }
  void rotate(const std::vector<double>& step) override {
    for (std::size_t i = 0; i < x_.size(); ++i) x_[i] += step[i];
  }
  void saveBest() override { best_ = x_; }
  void restoreBest() override { x_ = best_; }
  const std::vector<double>& x() const { return x_; }

 private:
  std::vector<double> a_, b_;
  double c_;
  std::vector<double> x_, best_;
};

}  // namespace

extern "C" {

// src/Utils/ADAM.cpp:33-51 Adam<T>::step over `nsteps` gradients (row t of grads / steps).
int rrref_adam_steps(i64 n, int cplx, i64 nsteps, double lr, double b1, double b2, double eps, const double* grads,
                     double* steps) {
  return guard([&] {
    const auto o = adamOptions(lr, b1, b2, eps);
    if (cplx) {
      rerdmft::Adam<C> adam(static_cast<std::size_t>(n), o);
      const C* g = reinterpret_cast<const C*>(grads);
      C* out = reinterpret_cast<C*>(steps);
      for (i64 t = 0; t < nsteps; ++t) {
        auto st = adam.step(std::vector<C>(g + t * n, g + (t + 1) * n));
        std::memcpy(out + t * n, st.data(), sizeof(C) * static_cast<std::size_t>(n));
      }
    } else {
      rerdmft::Adam<double> adam(static_cast<std::size_t>(n), o);
      for (i64 t = 0; t < nsteps; ++t) {
        auto st = adam.step(std::vector<double>(grads + t * n, grads + (t + 1) * n));
        std::memcpy(steps + t * n, st.data(), sizeof(double) * static_cast<std::size_t>(n));
      }
    }
  });
}

// src/Utils/ADAM.cpp:140-213 AdamOptimizer<double>::run, `runs` times in a row on QuadraticProblem.
// Per run: energy_best, iterations, restart flag, learning rate used; x_out: final point.
int rrref_adam_run_quadratic(i64 n, const double* a, const double* b, double c, const double* x0, int runs,
                             double* energy_best, int* iterations, int* restart, double* rate, double* x_out) {
  return guard([&] {
    QuadraticProblem prob(std::vector<double>(a, a + n), std::vector<double>(b, b + n), c,
                          std::vector<double>(x0, x0 + n));
    rerdmft::AdamOptimizer<double> opt;
    for (int r = 0; r < runs; ++r) {
      const auto res = opt.run(prob);
      energy_best[r] = res.energy_best;
      iterations[r] = res.iterations;
      restart[r] = res.restart_requested ? 1 : 0;
      rate[r] = res.learning_rate;
    }
    std::memcpy(x_out, prob.x().data(), sizeof(double) * static_cast<std::size_t>(n));
  });
}

// src/Hessian_opt/SpinorRotation.cpp:17 spinorRotationMatrix(kappa) = exp(-kappa).
int rrref_rotation_matrix(i64 n, int cplx, const double* kappa, double* U) {
  return guard([&] {
    if (cplx) fromCMatrix(rerdmft::spinorRotationMatrix(toCMatrix(kappa, n, n)), U);
    else fromMatrix(rerdmft::spinorRotationMatrix(toMatrix(kappa, n, n)), U);
  });
}

// src/Hessian_opt/OrbitalGradient.h orbitalGradient(F): g_pq = 2 (F_qp - conj F_pq), p >= q.
int rrref_orbital_gradient(i64 n, int cplx, const double* F, double* g) {
  return guard([&] {
    if (cplx) fromCMatrix(rerdmft::orbitalGradient(toCMatrix(F, n, n)), g);
    else fromMatrix(rerdmft::orbitalGradient(toMatrix(F, n, n)), g);
  });
}

// src/Hessian_opt/HartreeExchangeHessian.cpp:221 hartreeExchangeHessianElement(p,q,p,q) for each
// pair (p,q) of `pairs`, NON_REL spin-orbital RI tensor (RiNonRelSpinMoEri over n_sp spatial).
int rrref_hx_hessian_diag_nonrel(i64 n_sp, i64 naux, const double* Bmo, const double* h, const double* occ,
                                 const double* h2, const double* x2, const double* F, const i64* pair_of,
                                 const double* l1, const double* l2, i64 npairs, const i64* pairs, double* out) {
  return guard([&] {
    const i64 n = 2 * n_sp;
    rerdmft::RiNonRelSpinMoEri eri(static_cast<std::size_t>(n_sp), toMatrix(Bmo, naux, n_sp * n_sp));
    std::vector<double> o(occ, occ + n);
    Matrix<double> L1 = pair_of ? toMatrix(l1, n, n) : Matrix<double>();
    Matrix<double> L2 = pair_of ? toMatrix(l2, n, n) : Matrix<double>();
    const auto H = toMatrix(h, n, n), H2 = toMatrix(h2, n, n), X2 = toMatrix(x2, n, n), FF = toMatrix(F, n, n);
    const auto po = pairVec(pair_of, n);
    for (i64 i = 0; i < npairs; ++i) {
      const auto p = static_cast<std::size_t>(pairs[2 * i]), q = static_cast<std::size_t>(pairs[2 * i + 1]);
      out[i] = rerdmft::hartreeExchangeHessianElement(H, eri, o, H2, X2, FF, p, q, p, q, po, L1, L2);
    }
  });
}

// src/Hessian_opt/HartreeExchangeGradient.cpp:233 hartreeExchangeEnergy, NON_REL spin-orbital RI tensor.
int rrref_hx_energy_nonrel(i64 n_sp, i64 naux, const double* Bmo, const double* h, const double* occ,
                           const double* h2, const double* x2, const i64* pair_of, const double* l1, const double* l2,
                           double* E) {
  return guard([&] {
    const i64 n = 2 * n_sp;
    rerdmft::RiNonRelSpinMoEri eri(static_cast<std::size_t>(n_sp), toMatrix(Bmo, naux, n_sp * n_sp));
    std::vector<double> o(occ, occ + n);
    Matrix<double> L1 = pair_of ? toMatrix(l1, n, n) : Matrix<double>();
    Matrix<double> L2 = pair_of ? toMatrix(l2, n, n) : Matrix<double>();
    *E = rerdmft::hartreeExchangeEnergy(toMatrix(h, n, n), eri, o, toMatrix(h2, n, n), toMatrix(x2, n, n),
                                        pairVec(pair_of, n), L1, L2);
  });
}

}  // extern "C"
