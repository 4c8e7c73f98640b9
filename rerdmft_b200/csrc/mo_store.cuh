// Resident MO-basis RI tensor behind an rr_mo_handle.
#pragma once

#include "ri_store.cuh"

struct rr_mo_store {
  rr::Context ctx;
  int cplx = 0;          // 0: RiNonRelSpinMoEri (real spatial, accessors over 2n); 1: RiMoEri (complex)
  int64_t naux = 0, n = 0;
  rr::DevBuf<double> B;  // (naux, n*n) real, or complex interleaved
  // scratch
  rr::DevBuf<double> T, scratch, work, emb, hx, io;
};

namespace rr {
cudaStream_t mo_stream(rr_mo_store* m, const rr_opts* o);
void mo_build_nonrel(rr_ri_store* ri, const double* C, rr_mo_store* m, bool host, cudaStream_t s);
// RR_PREC_MIXED: the same tensor from split-BF16 tcgen05 products (mo_mixed.cu).
void mo_build_nonrel_mixed(rr_ri_store* ri, const double* C, rr_mo_store* m, bool host, cudaStream_t s);
void mo_build_ukb_mixed(rr_ri_store* ri, const double* c_ukb, int64_t nt, rr_mo_store* m, bool host, cudaStream_t s);
void mo_build_ukb(rr_ri_store* ri, const double* c_ukb, int64_t nt, rr_mo_store* m, bool host, cudaStream_t s);
void mo_rotate(rr_mo_store* src, const double* U, rr_mo_store* dst, bool host, cudaStream_t s);
void mo_positive_block(rr_mo_store* src, int64_t off, rr_mo_store* dst, cudaStream_t s);
void mo_embedded(rr_mo_store* m, double* out, bool host, cudaStream_t s);
void mo_eri(rr_mo_store* m, int64_t count, const int64_t* quads, double* out, bool host, cudaStream_t s);
void mo_jkl(rr_mo_store* m, const int64_t* pair_of, double* J, double* K, double* L, bool host, cudaStream_t s);
// The tensor the functional-stage operators act on: B itself (RiMoEri, d = n) or the block-diagonal
// embedded spin-orbital tensor in m->emb (RiNonRelSpinMoEri, d = 2n, the reference's embeddedB()).
const double* mo_operand(rr_mo_store* m, cudaStream_t s, int64_t* d);
// CASSCF RI operators (cas.cu).
void cas_two_electron(rr_mo_store* m, const double* rho, double* G, bool host, cudaStream_t s);
void cas_cumulant_fock(rr_mo_store* m, int64_t a, const int64_t* active, const double* lambda, double* F, bool host,
                       cudaStream_t s);
void cas_active_integrals(rr_mo_store* m, int64_t a, const int64_t* active, double* out, bool host, cudaStream_t s);
// hartreeExchangeJointHessianDiagonal on a complex tensor (hessian_joint.cu).
void mo_hx_joint_hessian_diagonal(rr_mo_store* m, const double* h, const double* occ, const double* h2,
                                  const double* x2, const double* fock, int64_t npairs, const int64_t* pairs,
                                  const int64_t* pair_of, const double* l1, const double* l2, double* out, bool host,
                                  cudaStream_t s);
void mo_hx_fock(rr_mo_store* m, const double* h, const double* occ, const double* h2, const double* x2,
                const int64_t* pair_of, const double* l1, const double* l2, double* F, bool host, cudaStream_t s);
}  // namespace rr
