// Split-BF16 operands and the tcgen05 exchange (RR_PREC_MIXED); see mixed_tc.cu.
#pragma once

#include "rr_common.cuh"

namespace rr {

struct MixedOperands {
  bool ready = false;
  int64_t n = 0, naux = 0, ldq = 0;
  DevBuf<uint16_t> bt_hi, bt_lo;  // resident: B^P transposed, split into BF16 hi/lo, [P][a][q], pitch ldq
  DevBuf<uint16_t> ct_hi, ct_lo;  // per call: occupied coefficients
  DevBuf<uint16_t> t_hi, t_lo;    // per call: half-transformed tensor, [a][P*nocc + i]
  DevBuf<float> work;             // split-K partial tiles
  DevBuf<double> kacc;
};

// Builds the resident split copy of B (rows of `pitch` doubles per aux index) once per store.
void mixed_prepare(MixedOperands& mo, const double* B, int64_t pitch, int64_t n, int64_t naux, cudaStream_t s);
// K (n x n FP64) = sum_P (Ct B^P)^T (Ct B^P) with Ct nocc x n (leading dim ldct) on the device.
void mixed_exchange(MixedOperands& mo, const double* Ct, int64_t ldct, int64_t nocc, double* K, int* err, cudaStream_t s);

}  // namespace rr
