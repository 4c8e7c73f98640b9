// Coulomb (J) streaming kernels over the resident RI tensor.
//   pass 1: gamma_P = sum_k B[P][k] * Dflat[k]          (reference: NonRelFockMatrixRi.cpp:88 DGEMV)
//   pass 2: J[k]    = sum_P gamma_P * B[P][k]           (reference: NonRelFockMatrixRi.cpp:91 DGEMV^T)
// Both passes stream B once from HBM through shared memory with 1-D TMA bulk copies
// (cp.async.bulk + mbarrier, one producer warp, 8 consumer warps) and reduce in a fixed order,
// so results are bit-identical run to run.  Up to two tensors (4c: LL and SS) share one gamma.
#pragma once

#include "rr_common.cuh"

namespace rr {

struct JTensor {
  const double* B = nullptr;  // (naux, pitch) rows, 256-byte aligned, zero padding beyond len
  int64_t pitch = 0;          // row pitch in doubles (multiple of 32)
  int64_t len = 0;            // valid entries per row (n^2)
  const double* D = nullptr;  // density, len entries (pass 1 input)
  double* J = nullptr;        // output, len entries (pass 2 output, written by j_finish)
};

struct JPlan {
  int ntens = 0;
  JTensor t[2];
  int64_t naux = 0;
  int nseg[2] = {0, 0};      // pass-1 segments per row of each tensor
  int nrange = 0;            // pass-2 aux ranges
  int64_t gpart_doubles = 0; // naux * (nseg[0] + nseg[1])
  int64_t jpart_doubles = 0; // nrange * (len[0] + len[1])
  int ctas_per_sm = 3;       // 1 when the passes share the GPU with concurrent GEMMs
};

JPlan j_plan(int ntens, const JTensor* t, int64_t naux, int ctas_per_sm = 3);

// gpart: plan.gpart_doubles scratch; jpart: plan.jpart_doubles scratch; err: device status word.
// skip (device int, may be null): when *skip != 0 at launch time the pass does nothing (the
// gamma partials were produced another way, decided on the device).
void j_pass1(const JPlan& plan, double* gpart, int* err, cudaStream_t s, const int* skip = nullptr);
// alt / alt_seg / alt_flag (optional): when *alt_flag != 0 at run time, gamma_P is summed from
// alt[P * alt_seg ...] instead of gpart.
void j_pass2(const JPlan& plan, const double* gpart, double* jpart, int* err, cudaStream_t s,
             const double* alt = nullptr, int alt_seg = 0, const int* alt_flag = nullptr);
// J[t][k] = scale * sum_r jpart[r][t][k]   (fixed order over r)
void j_finish(const JPlan& plan, const double* jpart, double scale, cudaStream_t s);

// Device pointer to the combined gamma vector is not materialised: pass 2 sums the pass-1 segments
// of each aux row itself.  j_gamma() exposes it for tests (naux doubles).
void j_gamma(const JPlan& plan, const double* gpart, double* gamma, cudaStream_t s);

}  // namespace rr
