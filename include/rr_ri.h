/* librr_ri — B200-native (sm_100a) RI two-electron hot path of ReRDMFT, C ABI.
 *
 * Drop-in boundary: the reference's C++ overload set keyed on the ERI-source struct
 * (src/NON_REL/NonRelFockMatrixRi.h:39, src/X2C_DHF/X2C_FockMatrixRi.h:38,
 * src/UKB/UkbFockMatrixRi.h:70 and :96, src/UKB/RiMoEri.h:91, src/NON_REL/NonRelSpinRiMoEri.h:101,
 * src/Hessian_opt/RiGemmFock.h:20-36).  The reference's source structs hold the 3-center tensor
 * by value; here it is uploaded ONCE into a handle and stays resident in HBM, and every call
 * passes only the small per-iteration matrices.  include/rr_ri.hpp re-creates the reference's
 * C++ overloads on top of these functions.
 *
 * Conventions
 *  - Matrices are row-major (the reference's Matrix<T>, src/Matrix.h:13).  Complex matrices are
 *    interleaved (re, im) doubles, i.e. std::complex<double> / numpy complex128 layout.
 *  - The RI tensor is (naux, n*n) row-major, B[P*n*n + m*n + k] = (mk|P)
 *    (src/AO_ints/ThreeCenterIntegrals.h:68 convention).
 *  - Every function returns RR_OK (0) or an RR_ERR_* code; rr_last_error() gives the message
 *    (thread-local).  Where the reference throws std::runtime_error on a dimension mismatch,
 *    the same condition returns RR_ERR_ARG.  No C++ exception crosses this boundary.
 *  - Pointer arguments live in host memory unless rr_opts.mem == RR_MEM_DEVICE (then they are
 *    device pointers on the handle's device).  Host outputs are complete on return.
 *  - A handle keeps its scratch (and the SCF loops' state) between calls, so one handle serves one
 *    call at a time; different handles may be used from different host threads at once (as
 *    rr_scf_run_x2c_batch does).
 */
#ifndef RR_RI_H
#define RR_RI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RR_OK 0
#define RR_ERR_ARG 1         /* invalid argument or dimension mismatch */
#define RR_ERR_CUDA 2        /* CUDA runtime error (message in rr_last_error) */
#define RR_ERR_SOLVER 3      /* eigensolver failure (reference: LAPACKE_* failed to converge) */
#define RR_ERR_TIMEOUT 4     /* a bounded device-side wait expired (kernel status word) */
#define RR_ERR_NOMEM 5       /* device allocation failed */
#define RR_ERR_STATE 6       /* handle in the wrong state for this call */
#define RR_ERR_UNSUPPORTED 7 /* option not supported by the library */

#define RR_MEM_HOST 0
#define RR_MEM_DEVICE 1

#define RR_PREC_FP64 0  /* every contraction in FP64 (DMMA tensor cores); matches the reference to ~1e-12 */
#define RR_PREC_MIXED 1 /* exchange contractions in split-BF16 (3 products, FP32 accumulate) on tcgen05 */

typedef struct rr_ri_store* rr_ri_handle;

/* Per-phase device times of the last profiled call (CUDA events on the streams that ran them). */
typedef struct rr_timings {
  double total_ms;          /* first to last event of the call, main stream */
  double recovery_ms;       /* occupied-orbital recovery: GEMMs + eigensolver (+ host readback) */
  double half_transform_ms; /* T[P] = C_occ^T B^P (batched FP64 DMMA, or split-BF16 tcgen05) */
  double exchange_ms;       /* K = sum_P T[P]^T T[P] (SYRK + split-K reduction) */
  double coulomb_ms;        /* J passes on the side stream (overlaps the exchange) */
  double epilogue_ms;       /* F assembly and output copies */
  double reserved[4];
} rr_timings;

typedef struct rr_opts {
  int32_t mem;       /* RR_MEM_HOST (default) or RR_MEM_DEVICE for every matrix argument of the call */
  int32_t precision; /* RR_PREC_FP64 (default) or RR_PREC_MIXED */
  void* stream;      /* cudaStream_t for the call; NULL = the handle's own stream */
  int32_t sync;      /* device-pointer calls: 1 = block until done (host-pointer calls always block) */
  int32_t incremental; /* RR_PREC_MIXED relativistic builds: 1 = add the split-BF16 exchange of the change of
                          the occupied spinors since the handle's previous mixed build (same rank), so the
                          rounding error scales with the density change; 0 = full split-BF16 exchange */
} rr_opts;

/* Message of the last failing call on this thread ("" if none). */
const char* rr_last_error(void);
/* Library version, major*10000 + minor*100 + patch. */
int rr_version(void);

/* Uploads the (naux, n*n) RI tensor once and keeps it resident in HBM.
 * Replaces constructing RiNonRelEriSource / RiX2cEriSource (src/NON_REL/NonRelFockMatrixRi.h:30,
 * src/X2C_DHF/X2C_FockMatrixRi.h:29): both hold eri3_L of this shape.  mem: RR_MEM_HOST or
 * RR_MEM_DEVICE for B.  The handle binds to the current CUDA device.  When every B^P is symmetric
 * to a few ulps and there is room (at most half of the free device memory), the handle also keeps
 * the packed upper triangles (naux * n(n+1)/2 doubles) for the Coulomb passes, which then stream
 * half of B; otherwise J streams B itself. */
int rr_ri_create(const double* B, int64_t naux, int64_t n, int32_t mem, rr_ri_handle* out);

/* 4-component variant: eri3_LL (naux, nl*nl) and eri3_SS (naux, ns*ns) sharing the aux index
 * (src/UKB/UkbFockMatrixRi.h:84 RiDirectEriSource).  Every B^P is taken to be symmetric, as an RI
 * tensor is: the relativistic builds write F's lower triangle from its upper one (F Hermitian), so a
 * B^P with asymmetry d changes F at order d. */
int rr_ri_create_4c(const double* B_LL, const double* B_SS, int64_t naux, int64_t nl, int64_t ns, int32_t mem,
                    rr_ri_handle* out);

int rr_ri_destroy(rr_ri_handle h);

/* ---------------- one-time set-up on the device ---------------- */

/* RankReductionReport (src/Linear_Algebra/LinearAlgebra.h). */
typedef struct rr_rank_report {
  int64_t n_kept, n_dropped;
  double smallest_kept, largest_dropped; /* 0 when nothing was kept / dropped (or all dropped are <= 0) */
} rr_rank_report;

/* canonicalOrthogonalize (hermitian = 0, real S) / canonicalOrthogonalizeHermitian (hermitian = 1,
 * interleaved complex S), src/Linear_Algebra/LinearAlgebra.cpp:267-349, on the device (cuSOLVER
 * eigensolver): the eigenvectors of S (of D^-1 S D^-1, D = diag(sqrt(Re S_ii)), for the Hermitian
 * form) whose eigenvalues exceed `threshold` (X_LIN_DEP_THRS_L / _S; 1e-10 for the aux metric), scaled
 * by 1/sqrt(eigenvalue) (and D^-1): X^dagger S X = I.  When nothing is dropped the real form returns
 * the symmetric S^-1/2 = U w^-1/2 U^T, as the reference does.  X must hold n*n elements; on return its
 * first n * n_eff elements are the n x n_eff matrix (row-major).  report may be NULL.  The reference
 * uses it for the AO overlaps (main.cpp:4476, 4544, 4584) and for the aux metric (X_metric,
 * src/AO_ints/ThreeCenterIntegrals.cpp:185-189).  Columns are determined up to sign / phase (and a
 * rotation inside a degenerate eigenvalue), as LAPACK's are. */
int rr_canonical_orthogonalize(const double* S, int64_t n, int32_t hermitian, double threshold, double* X,
                               int64_t* n_eff, rr_rank_report* report, const rr_opts* opts);

/* B = metric_x^T raw (naux_kept x n2): the metric contraction of riThreeCenterTensor,
 * src/AO_ints/ThreeCenterIntegrals.cpp:219-236, on the FP64 tensor cores.  raw: (naux_raw, n2) raw
 * 3-centre integrals (libcint's, from the host); metric_x: naux_raw x naux_kept (e.g. from
 * rr_canonical_orthogonalize of the aux metric). */
int rr_ri_three_center_tensor(const double* raw, int64_t naux_raw, int64_t n2, const double* metric_x,
                              int64_t naux_kept, double* B, const rr_opts* opts);

/* transformRiThreeCenterAoLegs, src/AO_ints/ThreeCenterIntegrals.cpp:191-217: B_out^P = t^T B_in^P t
 * per aux row (B_in: naux x n_ao^2, t: n_ao x n_out, B_out: naux x n_out^2), e.g. Cartesian ->
 * spherical / LOWGEN legs. */
int rr_ri_transform_ao_legs(const double* B_in, int64_t naux, int64_t n_ao, const double* t, int64_t n_out,
                            double* B_out, const rr_opts* opts);

/* A resident RI handle built on the device from the raw 3-centre integrals, as the reference builds its
 * source tensor (main.cpp:1108, 4922): B = metric_x^T raw (rr_ri_three_center_tensor), then, when t is
 * not NULL, t^T B^P t (rr_ri_transform_ao_legs; n = n_out), else n = n_ao.  The result is the handle
 * rr_ri_create would give for that B; mem applies to raw, metric_x and t. */
int rr_ri_create_raw(const double* raw, int64_t naux_raw, int64_t n_ao, const double* metric_x, int64_t naux_kept,
                     const double* t, int64_t n_out, int32_t mem, rr_ri_handle* out);

/* A list of contracted Cartesian Gaussian functions, the reference's std::vector<BasisFunction>
 * (src/AO_basis/MolecularBasis.h:13-22) flattened, in host memory: function i sits at center[3i..3i+2]
 * (bohr) with Cartesian exponents lxyz[3i..3i+2] (l = lx + ly + lz <= 6) and the primitives
 * [prim_offset[i], prim_offset[i+1]) of exponents / coefficients.  Coefficients are in libcint's
 * convention, as normalizeCartesianBasis (src/AO_ints/Integrals.cpp:140-187) leaves them: the function is
 * sum_p coefficient_p * f(l) * x^lx y^ly z^lz exp(-exponent_p r^2), f(0) = 1/sqrt(4 pi),
 * f(1) = sqrt(3/(4 pi)), f(l >= 2) = 1.  Runs of consecutive functions forming one shell in libcint's
 * component order (equal centre, l, exponents, proportional coefficients) are evaluated together. */
typedef struct rr_basis {
  int64_t n;
  const double* center;
  const int32_t* lxyz;
  const int64_t* prim_offset; /* n + 1 entries, prim_offset[0] = 0 */
  const double* exponents;
  const double* coefficients;
} rr_basis;

/* The aux metric (P|Q), naux x naux: auxMetric, src/AO_ints/ThreeCenterIntegrals.cpp:140-161 (libcint
 * cint2c2e_cart per shell pair there), on the GPU (McMurchie-Davidson, FP64).  opts->mem applies to
 * `metric`. */
int rr_int_aux_metric(const rr_basis* aux, double* metric, const rr_opts* opts);

/* The raw 3-centre integrals raw[P, p n + q] = (pq|P), naux x n^2: threeCenterIntegralsRaw,
 * src/AO_ints/ThreeCenterIntegrals.cpp:163-184 (libcint cint3c2e_cart there), on the GPU.  opts->mem
 * applies to `raw` (RR_MEM_DEVICE keeps the naux n^2 doubles on the device, e.g. for rr_ri_create_raw). */
int rr_int_three_center_raw(const rr_basis* basis, const rr_basis* aux, double* raw, const rr_opts* opts);

/* A resident RI handle from the basis sets alone, everything on the device: the aux metric, its canonical
 * orthogonalisation at metric_threshold (auxMetricOrthogonalization, ThreeCenterIntegrals.cpp:185-189;
 * the reference passes 1e-10, main.cpp:1085), the raw 3-centre integrals and riThreeCenterTensor's
 * contraction (:219-236), then t^T B^P t when t (host, n x n_out) is given, as rr_ri_create_raw.
 * naux_kept (may be NULL): the aux functions kept; report (may be NULL): the metric's rank report. */
int rr_ri_create_basis(const rr_basis* basis, const rr_basis* aux, double metric_threshold, const double* t,
                       int64_t n_out, rr_ri_handle* out, int64_t* naux_kept, rr_rank_report* report);

/* naux, n (nl for 4c) and ns (0 for a single-tensor handle). */
int rr_ri_info(rr_ri_handle h, int64_t* naux, int64_t* n, int64_t* ns);

/* Blocks until all work queued on the handle's streams is done; reports a device status error
 * (RR_ERR_TIMEOUT) left by an earlier asynchronous call. */
int rr_ri_sync(rr_ri_handle h);

/* Restricted nonrelativistic RI Fock matrix, F = h + J - K/2 (n x n, real).
 * Replaces nonRelFockMatrix(h_core, RiNonRelEriSource, D), src/NON_REL/NonRelFockMatrixRi.cpp:71:
 * D is the full (factor-2) density; the occupied orbitals are recovered from X^T (S D S / 2) X
 * (eigenvalues > 0.5) with the caller's X (n x n_eff) and S, exactly as the reference does. */
int rr_ri_fock_nonrel(rr_ri_handle h, const double* h_core, const double* D, const double* S, const double* X,
                      int64_t n_eff, double* F, const rr_opts* opts);

/* X2C RI Fock matrix in the [alpha; beta] spin-orbital AO basis (2nl x 2nl, complex).
 * Replaces x2cFockMatrix(h_x2c, RiX2cEriSource, P), src/X2C_DHF/X2C_FockMatrixRi.cpp:79: J from
 * Re(P_aa + P_bb) on both diagonal blocks, K over the two spin flavours from the occupied spinors
 * recovered from X^dagger (S P S) X (eigenvalues > 0.5, sqrt(eigenvalue)-weighted).  X: 2nl x n_eff.
 * opts->precision = RR_PREC_MIXED: K from the split-BF16 tcgen05 exchange (J stays FP64), full or
 * incremental (opts->incremental); the handle keeps the accumulated K between such calls. */
int rr_ri_fock_x2c(rr_ri_handle h, const double* h_x2c, const double* P, const double* S, const double* X,
                   int64_t n_eff, double* F, const rr_opts* opts);

/* Two-electron part in the UKB basis [L-alpha, L-beta, S-alpha, S-beta] (n_ukb = 2nl + 2ns,
 * complex) from P_ukb (J) and the caller's occupied coefficients C_occ (n_ukb x n_occ, complex) and
 * occupations (K).  Replaces riFockTwoElectronDirect, src/UKB/UkbFockMatrixRi.cpp:35. */
int rr_ri_two_electron_ukb(rr_ri_handle h, const double* P_ukb, const double* C_occ, int64_t n_occ,
                           const double* occupations, double* G, const rr_opts* opts);

/* 4-component RKB Fock matrix F = h + v^dagger G(v P v^dagger, v C_occ) v (n_rkb x n_rkb, complex).
 * Replaces rkbFockMatrix(h_rkb, RiDirectEriSource, P), src/UKB/UkbFockMatrixRi.cpp:185: the occupied
 * RKB spinors are recovered from x_full^dagger (s_full P s_full) x_full (eigenvalues > 0.5).
 * v_total: n_ukb x n_rkb; s_full: n_rkb x n_rkb; x_full: n_rkb x n_eff.  RR_PREC_MIXED as for
 * rr_ri_fock_x2c (the LL and SS exchange blocks on tcgen05). */
int rr_ri_fock_rkb(rr_ri_handle h, const double* h_rkb, const double* v_total, int64_t n_rkb, const double* s_full,
                   const double* x_full, int64_t n_eff, const double* P, double* F, const rr_opts* opts);

/* Coulomb and exchange from given occupied coefficients: J(D = 2 C C^T) and
 * K' = sum_P (C^T B^P)^T (C^T B^P) (so F = h + J - K'), C is n x n_occ.  The building block of
 * the device-resident SCF loop; equal to rr_ri_fock_nonrel when D = 2 C C^T. */
int rr_ri_jk_occupied(rr_ri_handle h, const double* C_occ, int64_t n_occ, double* J, double* K, const rr_opts* opts);

/* Coulomb matrix J = B^T (B vec D) (n x n, FP64) of a 2-component handle, computed with NO device
 * allocation: all scratch lives in one fixed 32 MiB device array inside the library (no
 * cudaMalloc, cudaFree or allocating library call on any path).  No counterpart in the reference:
 * it serves callers that cannot let the library allocate (a resident tensor that fills the device,
 * streams that a cudaFree would stall, a host that owns device memory through its own pool).
 *  - Sizes: round_up(n^2, 32) (copy of D) + round_up(n^2, 32) (J staging, host pointers only)
 *    + round_up(naux * s, 32) (pass-1 partials, s <= 64 segments per aux row) + n^2 (one pass-2
 *    range) doubles must fit in 4,194,304: n up to about 1150 with host pointers, 1400 with device
 *    pointers.  Larger sizes return RR_ERR_ARG with the required count, before any device work.
 *  - The first call on each device looks up the array's address (cudaGetSymbolAddress, which may
 *    load the module); make that first call before any stream capture on that device.
 *  - Nothing needs to be zeroed by the caller; the call clears the padding it reads.
 *  - There is one array per device: calls that overlap on one device (different streams or
 *    threads, any handles) race on it.  Order such calls on one stream or serialise them.
 *  - opts: mem, stream and sync as for the other calls; precision must be RR_PREC_FP64. */
int rr_ri_coulomb_noalloc(rr_ri_handle h, const double* D, double* J, const rr_opts* opts);

/* ---------------- device-resident SCF loops ---------------- */

typedef struct rr_scf_opts {
  int32_t diis_size;          /* DIIS_SIZE (reference default 5; < 2 disables DIIS) */
  int32_t max_iterations;     /* reference default 100 */
  double energy_tolerance;    /* ENERGY_TOLERANCE (1e-8) */
  double density_tolerance;   /* DENSITY_TOLERANCE (1e-6) */
  int32_t kramers_restricted; /* X2C / 4c: project densities onto their time-reversal-even part */
  int32_t precision;          /* RR_PREC_FP64 or RR_PREC_MIXED (split-BF16 exchange, FP64 for the last iterations) */
  double mixed_switch;        /* RR_PREC_MIXED: > 0 re-seeds the accumulated exchange once with an FP64
                                 build when |dE| < mixed_switch (0: never) */
  double mixing;              /* without DIIS (diis_size < 2): next density = mixing P_new + (1 - mixing) P,
                                 the reference's linear mixing; 0 is taken as 1 */
} rr_scf_opts;

typedef struct rr_scf_result {
  double electronic_energy; /* 1/2 Tr[P (h + F)] of the last iteration (no nuclear repulsion) */
  int64_t iterations;
  int64_t converged;
  int64_t mixed_iterations; /* Fock builds with the split-BF16 exchange */
  int64_t fp64_iterations;  /* Fock builds in FP64 */
  double seconds;           /* wall time of the loop, inputs on the device to density out */
  /* Device time per phase, summed over the iterations (only when rr_ri_set_profiling is on, else 0):
   * Fock builds (the final FP64 build of a mixed loop included), energy + DIIS, density step
   * (orthogonal transform, SP2 projector(s), back-transform, density change). */
  double build_ms, diis_ms, density_ms;
  /* Optional outputs, as the reference's SCF results carry them (src/NON_REL/NonRelHartreeFock.h:28-38,
   * src/X2C_DHF/X2C_HF.h:28-37, src/C4_DHF/C4_DHF.h:28-36).  The caller sets the pointers before the
   * call (NULL: not wanted; host or device memory as opts->mem says); the loop fills them from its last
   * iteration: orbital_energies (n_eff doubles, ascending) and c_matrix (C = X U, n x n_eff; complex for
   * X2C / DHF) from X^dagger F X = U diag(w) U^dagger, and fock_matrix (n x n) = that F: the
   * DIIS-extrapolated F of the last iteration, or, for a converged RR_PREC_MIXED loop, the FP64 Fock
   * matrix of the final density.  Eigenvectors are determined up to a phase per vector (and a rotation
   * within a degenerate level, e.g. a Kramers pair), as LAPACK's are. */
  double* orbital_energies;
  double* c_matrix;
  double* fock_matrix;
} rr_scf_result;

/* Restricted nonrelativistic SCF with the RI Fock build, DIIS on e = FPS - SPF and the aufbau
 * density from the lowest n_electrons/2 eigenvectors of X^T F X (obtained by SP2 purification on
 * the GPU).  Replaces runNonRelativisticHartreeFock(RiNonRelEriSource, ...),
 * src/NON_REL/NonRelHartreeFock.cpp:117-198/219 (nuclear repulsion is the caller's; DIIS replaces
 * the linear mixing as in the reference).  energy_history (optional) receives one electronic
 * energy per iteration (max_iterations doubles); P_out the density of the last iteration.
 * RR_PREC_MIXED: after the first (FP64) build, a full split-BF16 exchange, then builds adding the
 * split-BF16 exchange of the density change (J stays FP64); mixed_switch as for rr_scf_run_x2c; after
 * convergence one FP64 build of the final density gives the reported energy. */
int rr_scf_run_nonrel(rr_ri_handle h, const double* h_core, const double* X, int64_t n_eff, const double* S,
                      const double* P0, int32_t n_electrons, const rr_scf_opts* scf, rr_scf_result* result,
                      double* P_out, double* energy_history, const rr_opts* opts);

/* X2C-HF SCF on a 2-component handle: runX2CHartreeFockScf(h_x2c, RiX2cEriSource, x_large, P0,
 * n_electrons, ..., overlap, diis, ...), src/X2C_DHF/X2C_HF.cpp:43-138.  Complex interleaved
 * matrices: h_x2c, S, P0 (2nl x 2nl), X (2nl x n_eff).  Per iteration: F = x2cFockMatrix(P) on the
 * GPU, E = 1/2 Re Tr[P (h + F)], DIIS on e = FPS - SPF, P_new = X Pi X^dagger with Pi the SP2
 * projector onto the lowest n_electrons eigenvectors of X^dagger F X (one electron per spinor),
 * Kramers projection of every density ([alpha; beta] layout) when kramers_restricted and
 * n_electrons is even.
 * RR_PREC_MIXED: the first build uses the full split-BF16 exchange, later builds add the split-BF16
 * exchange of the density change (incremental); mixed_switch > 0 re-seeds the accumulated exchange
 * once with an FP64 build when |dE| < mixed_switch.  After convergence one FP64 build of the final
 * density gives the reported energy (counted in iterations and fp64_iterations). */
int rr_scf_run_x2c(rr_ri_handle h, const double* h_x2c, const double* X, int64_t n_eff, const double* S,
                   const double* P0, int32_t n_electrons, const rr_scf_opts* scf, rr_scf_result* result,
                   double* P_out, double* energy_history, const rr_opts* opts);

/* 4-component DHF SCF on a 4c handle: runDiracHartreeFockScf(h_rkb, RiDirectEriSource, x_full, P0,
 * n_electrons, ..., s_full, diis, ...), src/C4_DHF/C4_DHF.cpp:45-142.  Complex interleaved: h_rkb,
 * s_full, P0 (n_rkb x n_rkb), v_total (n_ukb x n_rkb), x_full (n_rkb x n_rkb: rkbDensityMatrix
 * needs the full basis).  F = rkbFockMatrix(P) on the GPU; the density fills the n_electrons
 * positive-energy spinors above the n_rkb/2 negative-energy ones (RkbDensityMatrix.cpp:16-43):
 * P_new = X (Pi_{n_rkb/2 + n_e} - Pi_{n_rkb/2}) X^dagger from two SP2 projectors; Kramers
 * projection in the [L-alpha; L-beta; S-alpha; S-beta] layout.  RR_PREC_MIXED as for
 * rr_scf_run_x2c. */
int rr_scf_run_dhf(rr_ri_handle h, const double* h_rkb, const double* v_total, int64_t n_rkb, const double* s_full,
                   const double* x_full, const double* P0, int32_t n_electrons, const rr_scf_opts* scf,
                   rr_scf_result* result, double* P_out, double* energy_history, const rr_opts* opts);

/* ---------------- MO-basis RI tensors (functional stage) ---------------- */

typedef struct rr_mo_store* rr_mo_handle;

#define RR_MO_NONREL_SPIN 0 /* RiNonRelSpinMoEri: real spatial tensor (naux, n*n); accessors span 2n spin orbitals */
#define RR_MO_COMPLEX 1     /* RiMoEri: complex tensor (naux, n*n) over n spinors */

/* buildRiNonRelSpinMoEri(eri3_L, n, C), src/NON_REL/NonRelSpinRiMoEri.cpp:13: B_mo^P = C^T B^P C
 * with the handle's resident eri3_L; C is n x n (the spatial alpha half of the coefficients).
 * opts->precision = RR_PREC_MIXED: both products as split-BF16 tcgen05 MMAs (three BF16 products, FP32
 * accumulation, the intermediate C^T B^P re-split to BF16 pairs), the tensor stored in FP64; relative
 * error about 1e-5 of max|B_mo| (the FP64 build is the default). */
int rr_mo_build_nonrel(rr_ri_handle ri, const double* C, rr_mo_handle* out, const rr_opts* opts);
/* The same build into an existing RR_MO_NONREL_SPIN tensor of the handle's naux and n, overwritten in
 * place (a functional-stage loop that rebuilds the tensor for new orbitals allocates nothing after the
 * first build); NonRelSpinRiMoEri.cpp:13-43 re-run on an existing object. */
int rr_mo_build_nonrel_into(rr_ri_handle ri, const double* C, rr_mo_handle mo, const rr_opts* opts);

/* buildRiMoEri(RiDirectEriSource, c_ukb), src/UKB/RiMoEri.cpp:64: B(P,p,q) = sum over the four UKB
 * blocks of sum conj(c(mu,p)) c(nu,q) (mu nu|P); c_ukb is n_ukb x n_total complex (n_ukb = 2nl+2ns
 * of a 4-component handle; an X2C handle is the ns = 0 case).  opts->precision = RR_PREC_MIXED: split-BF16
 * tcgen05 products as for rr_mo_build_nonrel (the four blocks and the real and imaginary parts in one K
 * range of 2 n_ukb), relative error about 1e-5 of max|B|. */
int rr_mo_build_ukb(rr_ri_handle ri4c, const double* c_ukb, int64_t n_total, rr_mo_handle* out, const rr_opts* opts);

/* Wraps an existing MO tensor (naux, n*n; kind RR_MO_NONREL_SPIN real or RR_MO_COMPLEX complex). */
int rr_mo_from_tensor(const double* Bmo, int64_t naux, int64_t n, int32_t kind, int32_t mem, rr_mo_handle* out);
int rr_mo_destroy(rr_mo_handle m);
/* naux, n (spatial orbitals for RR_MO_NONREL_SPIN, spinors for RR_MO_COMPLEX) and the kind. */
int rr_mo_info(rr_mo_handle m, int64_t* naux, int64_t* n, int32_t* kind);
/* Copies the tensor out (the reference's b()). */
int rr_mo_copy_tensor(rr_mo_handle m, double* out, const rr_opts* opts);

/* rotated(U): RiNonRelSpinMoEri::rotated (U 2n x 2n real, must be blockdiag(u,u) to 1e-3, the two
 * blocks are averaged; src/NON_REL/NonRelSpinRiMoEri.cpp:45) or RiMoEri::rotated (U n x n complex,
 * B' = U^dagger B U; src/UKB/RiMoEri.cpp:88).  A new handle is returned; m is unchanged. */
int rr_mo_rotated(rr_mo_handle m, const double* U, rr_mo_handle* out, const rr_opts* opts);

/* RiMoEri::positiveBlock(off), src/UKB/RiMoEri.cpp:112: both MO legs restricted to [off, n). */
int rr_mo_positive_block(rr_mo_handle m, int64_t off, rr_mo_handle* out, const rr_opts* opts);

/* RiNonRelSpinMoEri::embeddedB(), src/NON_REL/NonRelSpinRiMoEri.h:77: (naux, (2n)^2) block-diagonal. */
int rr_mo_embedded(rr_mo_handle m, double* out, const rr_opts* opts);

/* operator()(a,b,c,d) for `count` index quadruples (abcd: 4*count int64):
 * sum_P B(P,a,c) B(P,b,d) with the nonrelativistic spin selection rule where it applies
 * (src/NON_REL/NonRelSpinRiMoEri.h:40, src/UKB/RiMoEri.h:50).  out: count doubles or complex. */
int rr_mo_eri(rr_mo_handle m, int64_t count, const int64_t* abcd, double* out, const rr_opts* opts);

/* The functional stage's integral reads as whole matrices over the accessor dimension d
 * (2n or n): J_ij = eri(i,j,i,j), K_ij = eri(i,j,j,i) and, when pair_of (d int64) and L are given,
 * L_ij = eri(pair_of[i], j, j, pair_of[i]) (src/Occ_opt/PNOFs.cpp:306-321). */
int rr_mo_jkl(rr_mo_handle m, const int64_t* pair_of, double* J, double* K, double* L, const rr_opts* opts);

/* hartreeExchangeFockMatrix(h, eri, occupations, two_rdm_h, two_rdm_x, pair_of, l1, l2) GEMM form,
 * src/Hessian_opt/RiGemmFock.cpp:52-184 (riHxFockGemm; the nonrelativistic overload works on
 * embeddedB).  d = accessor dimension; h and F are d x d (complex for RR_MO_COMPLEX), occupations d,
 * two_rdm_* real d x d; pair_of may be NULL (no L terms; l1/l2 ignored). */
int rr_mo_hx_fock(rr_mo_handle m, const double* h, const double* occupations, const double* two_rdm_h,
                  const double* two_rdm_x, const int64_t* pair_of, const double* two_rdm_l1, const double* two_rdm_l2,
                  double* F, const rr_opts* opts);

/* hartreeExchangeJointHessianDiagonal (src/Hessian_opt/HartreeExchangeHessian.cpp:653-711, the RiMoEri
 * instantiation) on a complex MO tensor (RR_MO_COMPLEX, n spinors): out (2 n_pairs) = the diagonal of the
 * joint [real; imaginary] orbital-rotation Hessian for each pair (pairs: n_pairs x 2 int64 (p, q), p != q),
 * from h (complex n x n), the occupations, two_rdm_h / two_rdm_x (real n x n), fock (complex n x n, the
 * generalized Fock matrix of rr_mo_hx_fock) and optionally pair_of (n int64) with two_rdm_l1 / two_rdm_l2.
 * With a PNOF functional's full two-RDM (buildPnofFullTwoRdm / buildPnofPairOf) this is
 * pnofJointHessianDiagonal (src/Hessian_opt/PnofHessian.cpp:171-181).  The labels of the learned
 * preconditioner for complex orbitals.  A real tensor returns RR_ERR_UNSUPPORTED (no reference form). */
int rr_mo_hx_joint_hessian_diagonal(rr_mo_handle m, const double* h, const double* occupations,
                                    const double* two_rdm_h, const double* two_rdm_x, const double* fock,
                                    int64_t n_pairs, const int64_t* pairs, const int64_t* pair_of,
                                    const double* two_rdm_l1, const double* two_rdm_l2, double* out,
                                    const rr_opts* opts);

/* The CASSCF RI operators (src/MCSCF/CasFock.cpp:246-262) on an MO tensor; d = 2n for RR_MO_NONREL_SPIN
 * (the reference works on embeddedB()), n for RR_MO_COMPLEX; complex matrices interleaved.
 * casTwoElectronOperator: G (d x d) = J(rho) - K(rho) for a one-particle density rho (d x d), with K from
 * rho's eigen-decomposition (eigenvalues |w| > 1e-14, CasFock.cpp:74-113). */
int rr_mo_cas_two_electron(rr_mo_handle m, const double* rho, double* G, const rr_opts* opts);
/* casActiveCumulantFock (CasFock.cpp:116-133): F (d x n_active) = sum_r sum_P B(P, act[r], p)
 * T[P](r, q), T = Bact lambda with lambda[s, t, r, q] (n_active^4 entries); active: n_active indices in [0, d). */
int rr_mo_cas_cumulant_fock(rr_mo_handle m, int64_t n_active, const int64_t* active, const double* lambda, double* F,
                            const rr_opts* opts);
/* casActiveIntegrals (CasFock.cpp:136-147): (tu|vw) = sum_P B(P, t u) B(P, v w) over the active list,
 * n_active^4 values. */
int rr_mo_cas_active_integrals(rr_mo_handle m, int64_t n_active, const int64_t* active, double* out,
                               const rr_opts* opts);

/* One X2C-HF problem of a batch (its own 2-component handle and inputs, as for rr_scf_run_x2c);
 * result and status are outputs (status: RR_OK or the error code of this instance). */
typedef struct rr_x2c_instance {
  rr_ri_handle h;
  const double* h_x2c;
  const double* X;
  int64_t n_eff;
  const double* S;
  const double* P0;
  int32_t n_electrons;
  int32_t status;
  double* P_out;
  double* energy_history; /* optional */
  rr_scf_result result;
} rr_x2c_instance;

/* A batch of independent X2C-HF SCF problems of uneven size (a geometry scan) run concurrently:
 * `workers` host threads take the instances largest store first (naux * n^2, the cost of a build),
 * each instance running rr_scf_run_x2c on its
 * handle's own stream, so the small per-instance kernels of different instances overlap on the
 * GPU.  Host pointers.  Returns RR_OK when every instance succeeded, else the first failing
 * instance's code (all instances run; each reports its own status). */
int rr_scf_run_x2c_batch(rr_x2c_instance* instances, int64_t count, const rr_scf_opts* scf, int32_t workers);

/* The same batch in lockstep on one stream (the config-4 geometry scan as one grouped program):
 * every phase of an SCF iteration runs for all instances still iterating in one grouped launch
 * (persistent grouped FP64 DMMA GEMMs whose tile shapes and split-K counts come from the library's
 * autotuner, and grouped elementwise / reduction kernels), so the number of kernel launches per
 * iteration does not grow with the number of instances.  The first iteration takes the occupied
 * spinors from the caller's density in the same grouped form when that density is an idempotent
 * projector of the instance's n_electrons spinors, else by the single-instance recovery.  SP2 runs
 * from Gershgorin bounds.  FP64 only (RR_PREC_MIXED: RR_ERR_UNSUPPORTED); DIIS or linear mixing as
 * scf says.  Each instance's result does not depend on which other instances share the batch.  Host
 * pointers.  stats (optional) receives the batch's launch counts and times. */
typedef struct rr_batch_stats {
  int64_t iterations;             /* lockstep iterations (the largest instance count) */
  int64_t launches_total;         /* kernels launched by the call (autotuning excluded) */
  int64_t launches_setup;         /* of which before the first iteration's Fock build */
  int64_t launches_max_iteration; /* the most launched in one iteration */
  int64_t grouped_instances_first;/* instances whose first iteration ran grouped */
  double seconds;                 /* wall time of the call */
  double autotune_seconds;        /* of which spent timing new GEMM shapes */
  int64_t autotune_entries;       /* shapes in the autotuner cache afterwards */
  /* device time per phase summed over the iterations (CUDA events on the batch's stream): occupied
   * spinors + Fock build + energy, DIIS, density step (X^dagger F X, SP2, back-transform, dP) */
  double build_ms, diis_ms, density_ms;
  int64_t sp2_steps_max;          /* the most SP2 steps of one iteration */
  double host_wait_ms;            /* wall time the host spent waiting for the stream at read-backs */
  double host_gemm_ms;            /* wall time the host spent building and enqueueing grouped GEMMs */
} rr_batch_stats;

int rr_scf_run_x2c_grouped(rr_x2c_instance* instances, int64_t count, const rr_scf_opts* scf, rr_batch_stats* stats);

/* The grouped GEMM autotuner's cache: one line per problem shape ("<key> <configuration> <splits>
 * <microseconds per problem>").  The first tuning loads the file named by RR_AUTOTUNE_CACHE when that
 * variable is set, and rr_scf_run_x2c_grouped saves new entries there. */
int rr_autotune_load(const char* path);
int rr_autotune_save(const char* path);
int rr_autotune_clear(void);
int64_t rr_autotune_entries(void);

/* ---------------- RESTART files and the hand-over between runs of a scan ----------------
 * The reference's binary RESTART format (src/Utils/Restart.h:14-70), byte for byte: a file written by
 * rr_restart_write is read by the reference's readRestart and the other way round.  Strings are
 * NUL-terminated; vectors are pointer + count; coefficients are rows x cols row-major (interleaved
 * complex when complex_coefficients).  Version 3 is written; versions 2 and 3 are read. */
typedef struct rr_restart {
  const char* method;     /* "NON_REL" | "X2C" | "4C" */
  const char* functional; /* the FUNCTIONAL keyword */
  const char* kind;       /* "OCCUPATIONS" | "GAMMAS" | "PCCD" | "CASSCF" */
  uint64_t basis_fingerprint;
  int64_t n_electrons, pnof_subspaces, pnof_coupling, n_core, jk_frozen_pairs, jk_active_pairs;
  double total_energy;
  int32_t orbitals_optimized, converged;
  const double* occupations;
  int64_t n_occupations;
  const double* gammas;
  int64_t n_gammas;
  const double* amplitudes;
  int64_t n_amplitudes;
  int32_t complex_coefficients;
  int64_t rows, cols;
  const double* coefficients;
  int64_t cas_electrons, cas_spinors;
  const double* cas_state;
  int64_t n_cas_state;
} rr_restart;

/* writeRestart, src/Utils/Restart.cpp:94-145 (the same checks and messages).  Host only, no GPU. */
int rr_restart_write(const char* path, const rr_restart* data);
/* readRestart, src/Utils/Restart.cpp:147-197: fills *out with library-owned strings and arrays, which
 * rr_restart_release frees.  Host only, no GPU. */
int rr_restart_read(const char* path, rr_restart* out);
int rr_restart_release(rr_restart* data);
/* restartCoefficients, src/Utils/Restart.cpp:199-206: C = C_scf U on the GPU (C_scf rows x n_mo, U
 * n_mo x n_mo; U NULL = identity).  cplx: interleaved complex operands. */
int rr_restart_coefficients(const double* c_scf, int64_t rows, int64_t n_mo, const double* u, int32_t cplx,
                            double* c_out, const rr_opts* opts);
/* The starting density of the next run of a scan from a RESTART file's orbitals: P = C diag(occ) C^dagger
 * (rows x rows) on the GPU; for the SCF loops' conventions pass occupations 2 (RHF, spatial orbitals) or
 * 1 (spinors) on the occupied columns.  No counterpart in the reference, whose READ_RESTART path builds
 * the density on the host. */
int rr_density_from_orbitals(const double* C, int64_t rows, int64_t cols, const double* occupations, int32_t cplx,
                             double* P, const rr_opts* opts);

/* ---------------- RI sigma-vector Hessian-vector primitives (NEO orbital Hessian) ----------------
 * The GEMM engine behind the reference's RI Hessian-vector products (src/Hessian_opt/RiSigmaGemm.h,
 * src/Hessian_opt/RiSigmaHessianToolkit.h).  Tensors are (naux, n^2) row-major, element [P, i n + j];
 * cplx = 1: interleaved complex (RiMoEri's tensors), 0: real.  The real matrices (K, w, post, Wm) multiply
 * the complex values unconjugated, as in the reference.  All pointers host or device as opts->mem says. */

/* One operand of pairContract (RiSigmaGemm.h:21-41, PairOp): value(P, t, x) = [s ? s(P, idx[t n + x]) : 1]
 * * [w ? w[t n + x] : 1] * [row ? row(P, t) : 1], right-multiplied by `post` when given:
 * value(P, t, x) = sum_a v(P, t, a) post(a, x). */
typedef struct rr_pair_op {
  const double* s;      /* naux x n^2 (complex when cplx) or NULL */
  const uint32_t* idx;  /* n^2 indices into one row of s (needed with s) */
  const double* w;      /* n^2 real weights or NULL */
  const double* row;    /* naux x n (complex when cplx) or NULL */
  const double* post;   /* real n x n or NULL */
} rr_pair_op;

/* buildRiSigmaHessianToolkit(n, B, K), src/Hessian_opt/RiSigmaHessianToolkit.cpp:24-55: KB1[P] = K B^P,
 * KB2[P] = B^P K (naux x n^2 each) and Bdiag, KB1diag, KB2diag (naux x n each); K real n x n. */
int rr_sigma_toolkit(const double* B, int64_t n, int64_t naux, int32_t cplx, const double* K, double* kb1, double* kb2,
                     double* bdiag, double* kb1diag, double* kb2diag, const rr_opts* opts);

/* pairContract, src/Hessian_opt/RiSigmaGemm.cpp:65-95: target(x, y) += sign sum_{P,t} F(P,t,x) G(P,t,y)
 * (target n x n, in and out). */
int rr_sigma_pair_contract(double* target, double sign, int64_t n, int64_t naux, int32_t cplx, const rr_pair_op* f,
                           const rr_pair_op* g, const rr_opts* opts);

/* diagContract, src/Hessian_opt/RiSigmaGemm.cpp:97-114: target(a, b) += sum_P S(P, b n + a)
 * (Ua(P, a) + Ub(P, b)); Ua / Ub (naux x n) may be NULL. */
int rr_sigma_diag_contract(double* target, int64_t n, int64_t naux, int32_t cplx, const double* S, const double* Ua,
                           const double* Ub, const rr_opts* opts);

/* accumU, src/Hessian_opt/RiSigmaGemm.cpp:116-126: U(P, x) += alpha sum_t D[P n + t] Wm(x, t)
 * (U, D: naux x n; Wm real n x n). */
int rr_sigma_accum_u(double* U, double alpha, int64_t n, int64_t naux, int32_t cplx, const double* D, const double* Wm,
                     const rr_opts* opts);

/* ---------------- orbital-rotation optimisation (functional stage) ---------------- */

/* AdamOptions, src/Utils/ADAM.h:41-60 (rr_adam_default_options fills the reference's defaults). */
typedef struct rr_adam_options {
  double learning_rate;         /* 0.01 */
  double rate_factor;           /* 0.2: learning_rate *= rate_factor after a run that did not improve */
  double beta1, beta2, epsilon; /* 0.7, 0.9, 1e-15 */
  int32_t base_iterations;      /* 10 */
  int32_t iterations_increment; /* 20 */
  int32_t max_iterations_limit; /* 200 */
  int32_t reserved;
  double gradient_tolerance; /* 1e-5 */
  double energy_tolerance;   /* 1e-9 */
} rr_adam_options;

/* AdamResult, src/Utils/ADAM.h:182-197. */
typedef struct rr_adam_result {
  int32_t improved, gradient_converged, energy_converged, restart_requested;
  int32_t iterations, reserved;
  double energy_start, energy_best, energy_difference, max_gradient, learning_rate;
} rr_adam_result;

typedef struct rr_orbopt_store* rr_orbopt_handle;

int rr_adam_default_options(rr_adam_options* out);

/* The ADAM orbital-rotation problem of FULL_OPTIMIZATION (RotationProblem,
 * src/Full_opt/FullOptimization.cpp:1330-1548, with AdamOptimizer, src/Utils/ADAM.cpp:133-213) for a
 * fixed-occupation hartree-exchange functional, all on the GPU.  The handle takes a copy of m's tensor.
 * Nonrelativistic m (RR_MO_NONREL_SPIN): h is the n x n spatial one-electron matrix in m's MO basis,
 * occupations span the 2n spin orbitals, two_rdm_h / two_rdm_x are 2n x 2n, optional pair_of (2n)
 * with two_rdm_l1 / two_rdm_l2 (2n x 2n); pairs are adamPairIndices(2n) (p > q) and the spin-twin
 * pairs get the averaged gradient, so every rotation is spin restricted.
 * Complex m (RR_MO_COMPLEX, n spinors): h is n x n complex (interleaved), occupations n, the two-RDM
 * factors n x n real, optional pair_of (n) with l1 / l2; pairs are adamPairIndices(n) (p > q),
 * gradients, steps and rotations complex (RotationProblem<std::complex<double>>).
 * options NULL = the reference defaults. */
int rr_orbopt_create(rr_mo_handle m, const double* h, const double* occupations, const double* two_rdm_h,
                     const double* two_rdm_x, const int64_t* pair_of, const double* two_rdm_l1,
                     const double* two_rdm_l2, const rr_adam_options* options, rr_orbopt_handle* out);
/* Complex problems only: drop every pair that touches one of the first n_negative spinors (the
 * negative-energy branch of a 4-component basis) from the rotation (RotationProblem's n_negative,
 * excludeNegative, FullOptimization.cpp:83-92).  Clears the scales of rr_orbopt_set_scales. */
int rr_orbopt_exclude_negative(rr_orbopt_handle h, int64_t n_negative);
int rr_orbopt_destroy(rr_orbopt_handle h);
/* New occupations and two-RDM factors (the same shapes as at creation) for the next runs, as the macro
 * loop of FULL_OPTIMIZATION hands the re-optimised occupations to the orbital stage
 * (FullOptimization.cpp:2822-2835); the orbitals, the ADAM state and the scales are kept. */
int rr_orbopt_set_functional(rr_orbopt_handle h, const double* occupations, const double* two_rdm_h,
                             const double* two_rdm_x, const int64_t* pair_of, const double* two_rdm_l1,
                             const double* two_rdm_l2);
/* J_ij = eri(i,j,i,j) and K_ij = eri(i,j,j,i) of the current (rotated) tensor over the accessor's
 * dimension (2n spin orbitals, or n spinors, interleaved complex), host outputs: what the occupation
 * step reads (RiMoEri.h:50-57). */
int rr_orbopt_jk(rr_orbopt_handle h, double* J, double* K);
int rr_orbopt_info(rr_orbopt_handle h, int64_t* n_pairs, int64_t* n_spatial, int64_t* naux);
/* One AdamOptimizer::run: ADAM steps from the current orbitals until the gradient or energy
 * converges or the run's step budget ends; the best orbitals found become current.  The learning
 * rate, the extra-iteration allowance and the restart flag persist between runs, as in the
 * reference. */
int rr_orbopt_run(rr_orbopt_handle h, rr_adam_result* result);
/* Energy 1/2 sum_q [n_q Re h_qq + Re F_qq] and the pair gradient (n_pairs entries, interleaved complex
 * for a complex problem) at the current orbitals. */
int rr_orbopt_energy(rr_orbopt_handle h, double* energy);
int rr_orbopt_gradient(rr_orbopt_handle h, double* gradient);
/* Per-pair preconditioning scales s (n_pairs, positive; NULL = plain ADAM): ADAM sees g / sqrt(s)
 * and the rotation uses step / sqrt(s), the variable change the reference's min-max stage applies
 * (FullOptimization.cpp:1362-1369).  No counterpart for the learned use in the reference. */
int rr_orbopt_set_scales(rr_orbopt_handle h, const double* scales);
/* hartreeExchangeHessianElement(p,q,p,q) per pair at the current orbitals
 * (src/Hessian_opt/HartreeExchangeHessian.cpp:221), the labels of the learned preconditioner; for a
 * complex problem the joint [t; y] diagonal of hartreeExchangeJointHessianDiagonal over the pairs
 * (2 n_pairs entries). */
int rr_orbopt_hessian_diagonal(rr_orbopt_handle h, double* out);
/* Preconditioner inputs per pair (i = q, a = p): F_ii, F_aa, n_i, n_a, J_ia, K_ia, J_ii, J_aa
 * (n_pairs x 8 floats; F the generalized Fock matrix, J/K the MO Coulomb and exchange integrals;
 * real parts for a complex problem). */
int rr_orbopt_features(rr_orbopt_handle h, float* out);
/* Current accumulated rotation (n x n), rotated h (n x n) and MO tensor (naux x n^2), interleaved
 * complex for a complex problem; any pointer may be NULL. */
int rr_orbopt_state(rr_orbopt_handle h, double* rotation, double* h_out, double* Bmo_out);

/* ---------------- learned preconditioner (no counterpart in the reference) ----------------
 * An 8 -> 64 -> 64 -> 64 -> 1 tanh MLP predicting log |hartreeExchangeHessianElement(p,q,p,q)| from the
 * rr_orbopt_features inputs; trained in FP32 by the library's own kernels, BF16 inference.  Its
 * predictions become rr_orbopt_set_scales scales; without it the optimiser is plain ADAM. */
typedef struct rr_mlp_store* rr_mlp_handle;
#define RR_MLP_PARAMS 8961 /* W1 64x8, b1, W2 64x64, b2, W3 64x64, b3, W4 1x64, b4 (row-major, in that order) */
#define RR_MLP_NORM 18     /* input mean[8], input spread[8], label mean, label spread */

int rr_mlp_create(uint64_t seed, rr_mlp_handle* out); /* Xavier-uniform weights from the seed */
int rr_mlp_destroy(rr_mlp_handle h);
/* Mini-batch Adam (beta 0.9 / 0.999) on the mean squared error of the standardised labels; the
 * first call fixes the input / label standardisation from its data.  X: count x 8, y: count (host).
 * loss_per_epoch (optional): mean squared error per epoch, in standardised units. */
int rr_mlp_train(rr_mlp_handle h, const float* X, const float* y, int64_t count, int32_t epochs, int32_t batch,
                 float learning_rate, uint64_t shuffle_seed, float* loss_per_epoch);
/* y = prediction in label units; bf16 != 0 runs the BF16 inference kernel, else FP32. */
int rr_mlp_predict(rr_mlp_handle h, const float* X, int64_t count, int32_t bf16, float* y);
/* Loss (mean squared error, standardised units) and its gradient (RR_MLP_PARAMS floats) over all
 * `count` samples: the training kernels' forward and backward passes, for gradient checks. */
int rr_mlp_loss_and_grad(rr_mlp_handle h, const float* X, const float* y, int64_t count, float* loss, float* grad);
/* RR_MLP_PARAMS weights followed by the RR_MLP_NORM standardisation constants. */
int rr_mlp_get_params(rr_mlp_handle h, float* params);
int rr_mlp_set_params(rr_mlp_handle h, const float* params);

/* Profiling: when on, each call records CUDA events around its phases; rr_ri_get_timings waits
 * for the last call's events and returns the phase times.  Off by default (no event overhead). */
int rr_ri_set_profiling(rr_ri_handle h, int32_t on);
int rr_ri_get_timings(rr_ri_handle h, rr_timings* out);

/* Number of librr_ri kernel launches issued by this process so far (library kernels such as the
 * cuSOLVER eigensolver are not counted). */
int64_t rr_kernel_launches(void);

#ifdef __cplusplus
}
#endif

#endif /* RR_RI_H */
