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
  int64_t len = 0;            // valid entries per row (n^2, or n(n+1)/2 packed)
  const double* D = nullptr;  // density, len entries (pass 1 input; packed rows: j_fold_density)
  double* J = nullptr;        // output, len entries (n^2 for packed rows), written by j_finish
  int64_t tri_n = 0;          // > 0: rows hold the packed upper triangles of symmetric tri_n x tri_n B^P
};

// Packed upper triangle of a symmetric n x n matrix, row by row: (q, a >= q) -> tri_index.
__host__ __device__ inline int64_t tri_len(int64_t n) { return n * (n + 1) / 2; }
__host__ __device__ inline int64_t tri_index(int64_t q, int64_t a, int64_t n) { return q * (2 * n - q + 1) / 2 + (a - q); }

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

// The reference's three-centre tensor is symmetric in its two AO indices
// (src/AO_ints/ThreeCenterIntegrals.cpp:177-178), so half of each row carries all of it.
// Packs the upper triangles of the naux n x n rows of B (row pitch `pitch`) into `out`, row pitch
// pitch_out = round_up(tri_len(n), 32), zero padded.  Every B^P must be symmetric to a few ulps
// (|B_qa - B_aq| <= 8 eps max(|B_qa|, |B_aq|)): then gamma_P = sum_{q<=a} B^P_qa (D_qa + D_aq [a != q])
// and J_qa = J_aq = sum_P gamma_P B^P_qa equal the full passes up to rounding, and the passes stream
// half of B.  Returns false and releases `out` when some element fails the test.  Synchronises s.
bool j_pack_upper(const double* B, int64_t pitch, int64_t naux, int64_t n, DevBuf<double>& out, int64_t& pitch_out,
                  cudaStream_t s);
// Dpk[tri_index(q, a)] = D_qa + D_aq (a > q), D_qq (a == q) for the n x n row-major D; Dpk holds
// round_up(tri_len(n), 2) entries (an odd length gets a zero pad for the 16-byte loads of pass 1).
void j_fold_density(const double* D, int64_t n, double* Dpk, cudaStream_t s);

// Device pointer to the combined gamma vector is not materialised: pass 2 sums the pass-1 segments
// of each aux row itself.  j_gamma() exposes it for tests (naux doubles).
void j_gamma(const JPlan& plan, const double* gpart, double* gamma, cudaStream_t s);

}  // namespace rr
