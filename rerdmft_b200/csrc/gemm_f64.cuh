// FP64 tensor-core GEMM family (DMMA, mma.sync m8n8k4 .f64) used by every FP64 contraction of
// the RI path: half-transforms, the exchange SYRK, the occupied recovery products, the MO
// transforms and the generalized-Fock contraction.  tcgen05 has no FP64 kind, so the FP64
// tensor pipe is reached through DMMA; the BF16 split path lives in mixed_tc.cu.
//
// Row-major semantics throughout (the reference's Matrix<T> layout):
//   C[b] = alpha * op(A[b]) * op(B[b]) + beta * C[b],  op(A): M x K,  op(B): K x N,
// with op in {N, T} and optional element conjugation for complex (interleaved re,im) operands.
#pragma once

#include "rr_common.cuh"

namespace rr {

enum class Op : int { N = 0, T = 1 };

struct GemmDesc {
  int64_t M = 0, N = 0, K = 0;
  const double* A = nullptr;
  int64_t lda = 0, strideA = 0;  // in elements (complex elements when cplx)
  const double* B = nullptr;
  int64_t ldb = 0, strideB = 0;
  double* C = nullptr;
  int64_t ldc = 0, strideC = 0;
  Op opA = Op::N, opB = Op::N;
  double alpha = 1.0, beta = 0.0;
  int64_t batch = 1;
  bool cplx = false;
  bool conjA = false, conjB = false;
  // Output rows r >= c_plane_rows go to C + (r / c_plane_rows) * c_plane_stride, row r % c_plane_rows
  // (0 disables).  Lets one GEMM write the stacked [re; im] half-transform into two planes.
  int64_t c_plane_rows = 0, c_plane_stride = 0;
  // Element stride between consecutive output columns (real outputs only; 2 with c_plane_stride = 1
  // and c_plane_rows = M/2 writes a stacked [re; im] product as interleaved complex).
  int64_t c_col_stride = 1;
  // Symmetric outputs: compute only tiles touching the upper triangle, then fill the strict
  // lower triangle from the upper one: +1 C[i][j] = C[j][i] (Hermitian conj for cplx),
  // -1 C[i][j] = -C[j][i].  0 = full output.  Requires M == N.  2 (grouped GEMM only): the upper
  // tiles and nothing else; the strict lower triangle is left for the consumer to read as the mirror.
  int mirror = 0;
  // Epilogue dot (real, no split-K): per output tile also
  //   edot_out[b * tiles + tile] = edot_scale * sum_{(m,n) in tile} C[b](m, n) * edot_E[m * edot_ld + n]
  // with tiles = (output tile columns) x (output tile rows), tile = ty * tiles_x + tx.
  const double* edot_E = nullptr;
  int64_t edot_ld = 0;
  double edot_scale = 1.0;
  double* edot_out = nullptr;
};

// Output tiles per batch entry gemm() uses for this descriptor (size of an edot segment).
int64_t gemm_tiles_per_batch(const GemmDesc& d);

// Launches the GEMM on `stream`.  `work` (capacity `work_cap` doubles) is split-K scratch: when
// the output grid is too small to fill the GPU and work_cap allows, K is split, the partial
// products go to `work` and a deterministic fixed-order reduction finishes C.  work may be null.
void gemm(const GemmDesc& d, cudaStream_t stream, double* work = nullptr, int64_t work_cap = 0);

// Doubles of scratch gemm() would like for split-K on this descriptor.
int64_t gemm_work_doubles(const GemmDesc& d);

// T[P] = Ct B^P for P < naux on the m16n8k8 FP64 shape (ht_dmma16.cu): Ct nocc x n (row pitch n), B^P
// n x n in rows of `pitch` doubles, T[P] at T + P nocc n (row pitch n).  Returns false (nothing launched)
// when the operands do not meet its 16-byte alignment rule.  config 0 is the default tiling (2 warps,
// 16-deep k tiles, 3 stages); 1-6 are the alternatives kept for measurement: (warps, k depth, stages) =
// (1,16,4), (2,16,4), (5,32,2), (4,16,3), (1,32,3), (2,32,3); 7 and 8 the warp-specialised bulk-copy
// pipeline with 4 and 3 stages (they need `status`, the device word a timed-out wait sets); 9-13:
// (2,16,5), (5,16,3), (2,16,6), (4,16,4), (3,16,4).
bool half_transform_m16(const double* Ct, int64_t nocc, const double* B, int64_t pitch, int64_t naux, int64_t n,
                        double* T, cudaStream_t s, int config = 0, int* status = nullptr);
// Which half-transform the nonrelativistic exchange uses: 0 = the general DMMA GEMM (m8n8k4),
// 1 = half_transform_m16 (the default).  RR_HALF_TRANSFORM=m8|m16 overrides the default.
int half_transform_kind();
// The m16 tiling the exchange uses (config of half_transform_m16): 0 unless RR_HALF_TRANSFORM=m16:<config>
// names another (for measurement).
int half_transform_config();

}  // namespace rr
