// Split-BF16 operands and the tcgen05 exchange (RR_PREC_MIXED); see mixed_tc.cu.
#pragma once

#include <cuda.h>

#include "rr_common.cuh"

namespace rr {

// Resident split copy of one 3-centre tensor: B^P transposed, split into BF16 hi/lo, [P][a][q],
// row pitch ldq (built once per store on the first mixed call).
struct MixedOperands {
  bool ready = false;
  int64_t n = 0, naux = 0, ldq = 0;
  DevBuf<uint16_t> bt_hi, bt_lo;
};

// Per-call scratch of the split-BF16 exchange, grown on demand: coefficient rows of one
// half-transform pass, the half-transformed output planes of every flavour, split-K partials.
struct MixedScratch {
  DevBuf<uint16_t> coef_hi, coef_lo;
  DevBuf<uint16_t> pl_hi, pl_lo;
  DevBuf<float> work;
  DevBuf<double> xacc;  // incremental builds: X = sum_P (W B^P)^dagger (U B^P) before K += X + X^dagger
};

// Flavour blocks of the exchange: columns [off, off + fs) of c_t contract with tensor `tens`.
// Nonrelativistic: one flavour.  X2C: alpha / beta on one tensor.  4c: L alpha, L beta on the LL
// tensor and S alpha, S beta on the SS tensor.
struct ExFlavours {
  int nf = 0;
  int64_t off[4] = {0, 0, 0, 0}, fs[4] = {0, 0, 0, 0};
  int tens[4] = {0, 0, 0, 0};
};

// Builds the resident split copy of B (rows of `pitch` doubles per aux index) once per store.
void mixed_prepare(MixedOperands& mo, const double* B, int64_t pitch, int64_t n, int64_t naux, cudaStream_t s);

// Split-BF16 exchange on tcgen05 for every flavour block (f, u):
//   K_fu = sum_P (Ct_f B^P)^dagger (Ct_u B^P)                         (Ct_prev == nullptr)
//   K_fu = X_fu + X_uf^dagger,  X_fu = sum_P (W_f B^P)^dagger (U_u B^P),
//          W = (Ct + Ct_prev) / 2, U = Ct - Ct_prev                    (Ct_prev given)
// The second form is exactly K(Ct) - K(Ct_prev), with a rounding error proportional to |U|
// instead of |Ct|.  Ct / Ct_prev: r x ld row-major, real or interleaved complex (cplx).  K: real or
// interleaved complex, leading dimension ldk; f < u blocks also fill their (u, f) mirror.  With
// accumulate the blocks are added to K, otherwise K (ldk x ldk) is overwritten.
void mixed_exchange_general(const MixedOperands* ops, MixedScratch& scr, const ExFlavours& fl, int64_t naux,
                            const double* Ct, const double* Ct_prev, int64_t ld, int64_t r, bool cplx, double* K,
                            int64_t ldk, bool accumulate, int* err, cudaStream_t s);

// Nonrelativistic K (n x n FP64, symmetric) = sum_P (Ct B^P)^T (Ct B^P), Ct nocc x n (leading dim
// ldct) on the device.
void mixed_exchange(const MixedOperands& mo, MixedScratch& scr, const double* Ct, int64_t ldct, int64_t nocc, double* K,
                    int* err, cudaStream_t s);

// BF16 tensor map with a 128- or 64-byte swizzle and zero fill out of bounds; dims / strides (bytes,
// rank-1 entries) / box innermost first.
CUtensorMap bf16_tensor_map(const void* base, int rank, const uint64_t* dims, const uint64_t* strides_bytes,
                            const uint32_t* box, int swizzle_bytes = 128);

}  // namespace rr
