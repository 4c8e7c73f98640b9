// The resident RI store behind an rr_ri_handle, and the helpers every entry point shares.
#pragma once

#include "gemm_f64.cuh"
#include "j_stream.cuh"
#include "mixed.cuh"
#include "rr_common.cuh"

struct rr_ri_store {
  rr::Context ctx;
  int64_t naux = 0, n = 0, ns = 0;  // n = nl for the 4c store
  int ntens = 1;
  rr::DevBuf<double> B[2];  // resident tensors, row pitch `pitch` doubles (256-byte aligned rows)
  int64_t pitch[2] = {0, 0};
  // Packed upper triangles of B[t] (rr::j_pack_upper), built at creation when every B^P is
  // symmetric and the copy fits in half of the free memory; the J passes then stream these.
  rr::DevBuf<double> Bpk[2];
  int64_t pitch_pk[2] = {0, 0};
  rr::DevBuf<int> status;   // device status word written by bounded waits
  // Scratch, grown on demand and reused across calls.
  rr::DevBuf<double> mats;  // per-call matrices (inputs, outputs, intermediates)
  rr::DevBuf<double> T;     // half-transformed exchange intermediate
  rr::DevBuf<double> kpart; // per-chunk exchange partials of the pipelined half-transform / SYRK
  rr::DevBuf<double> work;  // split-K partial products
  rr::DevBuf<double> jscr;  // J pass-1/pass-2 partial sums
  rr::DevBuf<double> dfold; // densities folded onto the packed triangles
  // Coulomb passes prepared by coulomb_prep and launched by coulomb_run.
  struct {
    rr::JPlan pl;
    double *gpart = nullptr, *jpart = nullptr;
    int* flag = nullptr;
    cudaStream_t s = nullptr;
    bool overlap = false;
  } jpend;
  rr::DevBuf<double> tgam;  // gamma partials from the half-transform epilogue
  rr::DevBuf<double> solver_a;  // eigen-problem matrix / eigenvectors
  // SCF loop state (matrices, DIIS history), grown on demand and kept with the handle, so that
  // repeated SCF runs allocate nothing (a cudaFree would synchronise the whole device, and with
  // it every other thread's handle).
  rr::DevBuf<double> scf_buf, diis_err, diis_val, diis_dots;
  rr::DevBuf<double> solver_w;  // eigenvalues
  std::vector<double> host_w;
  // Split-BF16 copies of B[t] for RR_PREC_MIXED (built on first use) and their call scratch.
  rr::MixedOperands mixed[2];
  rr::MixedScratch mscr;
  // Incremental (density-change) builds of the mixed SCF loops: the exchange accumulated so far
  // (n x n real, or ntot x ntot interleaved complex) and the c_t it belongs to (inc_r rows of
  // inc_ld entries).
  rr::DevBuf<double> inc_k, inc_ct;
  int64_t inc_r = -1, inc_ld = 0;
  // Host waits of the SCF loops: blocking (the waiting thread sleeps on an event) when many host
  // threads drive handles at once (rr_scf_run_x2c_batch), spinning stream syncs otherwise.
  bool blocking_wait = false;
  cudaEvent_t wait_ev = nullptr;
  // Profiling events: 0 start, 1 recovery done, 2 half-transform done, 3 exchange done, 4 end
  // (main stream); 5 J start, 6 J end (side stream).
  bool profiling = false;
  cudaEvent_t ev[8] = {};
  bool ev_used[8] = {};
};

namespace rr {

// Bump allocator over a DevBuf<double>: carve(n) returns 256-byte-aligned sub-buffers.
struct Arena {
  DevBuf<double>* buf;
  int64_t used = 0;
  std::vector<std::pair<double**, int64_t>> pending;
  explicit Arena(DevBuf<double>* b) : buf(b) {}
  // Two-phase: request() records sizes, commit() grows the buffer once and fills pointers.
  void request(double** p, int64_t count) {
    pending.emplace_back(p, count);
    used += round_up(std::max<int64_t>(count, 1), 32);
  }
  void commit() {
    buf->ensure(static_cast<size_t>(used));
    int64_t off = 0;
    for (auto& pr : pending) {
      *pr.first = buf->p + off;
      off += round_up(std::max<int64_t>(pr.second, 1), 32);
    }
    pending.clear();
  }
};

// How a relativistic Fock build forms its exchange.  nullptr: FP64, straight into G.  Otherwise the
// exchange goes through the handle's accumulator (inc_k), G = J - inc_k:
//   mixed:           split-BF16 exchange on tcgen05; with `incremental` (and a previous build of the
//                    same rank) only the exchange of c_t - c_t(previous) is added to inc_k, so the
//                    rounding error scales with the density change;
//   otherwise:       FP64 exchange that (re)seeds inc_k.
// energy (device, 2 doubles; not with mixed): energy-only FP64 evaluation, no G and no F: J in FP64 and
// the FP64 half-transform only, energy[0] = E_J = 1/2 sum_t <D_t, J_t> (spin-summed densities) and
// energy[1] = E_K = sum_P || sum_f c_f B^P c_f^dagger ||_F^2 = Re Tr[c_t^dagger c_t K], so that
// 1/2 Re Tr[P (h + F)] = Re Tr[P h] + E_J - E_K / 2 for P = c_t^dagger c_t; inc_k is left untouched.
struct RelBuild {
  bool mixed = false;
  bool incremental = false;
  double* energy = nullptr;
};

cudaStream_t call_stream(rr_ri_store* h, const rr_opts* o);
// Occupied-orbital recovery (recovery.cu): c_t (r x n) from the density; returns r.  d_ready
// (optional): event s waits on before the first product that reads Dp.
int64_t occupied_ct(rr_ri_store* h, const double* X, const double* S, const double* Dp, int64_t n, int64_t n_eff,
                    double scale, bool cplx, bool weighted, double* Ct, cudaStream_t s, cudaEvent_t d_ready = nullptr);
// Builds h->Bpk[t] from h->B[t] (n x n rows) when it fits; synchronises s.
void pack_for_j(rr_ri_store* h, int t, int64_t n, cudaStream_t s);
// JTensor of tensor t (n x n rows) over the packed copy when there is one (D folded into dfold at
// offset doff doubles) or over B[t] itself (D used as is).
JTensor j_tensor(rr_ri_store* h, int t, int64_t n, const double* D, double* J, int64_t doff, cudaStream_t s);
// Records profiling event i on stream s when profiling is on.
void prof_mark(rr_ri_store* h, int i, cudaStream_t s);
int64_t launches();
void sp2_projector(rr_ri_store* h, const double* F, int64_t n, int64_t nocc, double* Pi, double* T, double* scal,
                   cudaStream_t s, bool cplx = false);
void check_status(rr_ri_store* h, cudaStream_t s);  // syncs s, throws RR_ERR_TIMEOUT on a set word
// The DIIS bordered solve of the SCF loops (Gaussian elimination with partial pivoting; false when
// min |pivot| / max |pivot| is not above tol).
bool diis_solve(const std::vector<double>& m, const std::vector<double>& rhs, size_t n, double tol,
                std::vector<double>& x);
// Orbital energies, C and F of an SCF loop's last iteration into the result's output pointers.
void scf_result_outputs(rr_ri_store* h, const double* F, const double* Xd, int64_t n, int64_t n_eff, bool cplx,
                        const rr_scf_result* res, bool host, cudaStream_t s);
// Waits on the host for everything queued on s (see rr_ri_store::blocking_wait).
void host_wait(rr_ri_store* h, cudaStream_t s);
void copy_in(double* dst, const double* src, int64_t count, bool host, cudaStream_t s);
void copy_out(double* dst, const double* src, int64_t count, bool host, cudaStream_t s);
// Pitched copy of a flat n2-vector into a zero-padded buffer of `pitch` doubles.
void copy_in_padded(double* dst, int64_t pitch, const double* src, int64_t n2, bool host, cudaStream_t s);

// Elementwise helpers (device).
void axpby(double* y, const double* x, double a, double b, int64_t n, cudaStream_t s);  // y = a x + b y
// out (cols x rows) = in^T for a real row-major rows x cols matrix.
void transpose(double* out, const double* in, int64_t rows, int64_t cols, cudaStream_t s);
// out[0] (device) = scale * sum_k a[k] b[k] over cnt entries (sum of a[k]^2 when b is null), or
// out[0] += that with accumulate; deterministic (fixed-order two-stage sum), part: 256 doubles of scratch.
void dot_sum(const double* a, const double* b, int64_t cnt, double scale, double* out, bool accumulate, double* part,
             cudaStream_t s);
// F = h + J - K (real, n2 entries).
void fock_combine(double* F, const double* h, const double* J, const double* K, int64_t n2, cudaStream_t s);
// Symmetric eigensolver (cuSOLVER dsyevd) in place on a (n x n) row-major symmetric matrix:
// on return row j of `a` holds eigenvector j; w ascending.
void eigh_sym(rr_ri_store* h, double* a, int64_t n, double* w, cudaStream_t s);
// Hermitian (interleaved complex) version, cuSOLVER zheevd; row j of `a` holds conj(eigenvector j).
void eigh_herm(rr_ri_store* h, double* a, int64_t n, double* w, cudaStream_t s);
// The same on any execution context (its cuSOLVER handle and scratch); the info word is left in
// c.solver_info.
void eigh_sym_ctx(Context& c, double* a, int64_t n, double* w, cudaStream_t s);
void eigh_herm_ctx(Context& c, double* a, int64_t n, double* w, cudaStream_t s);
// canonicalOrthogonalize(Hermitian) on the device (tensor_build.cu): X (n x n_eff, caller's n x n buffer),
// opts->mem for S and X, opts->stream (or a private stream) for the work.
void canonical_orthogonalize(const double* S, int64_t n, bool herm, double threshold, double* X, int64_t* n_eff_out,
                             rr_rank_report* report, const rr_opts* o);

}  // namespace rr
