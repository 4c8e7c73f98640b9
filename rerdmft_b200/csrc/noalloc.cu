// Coulomb matrix from the resident RI tensor with no device allocation at call time.
//
// rr_ri_fock_nonrel and the other entry points grow per-handle scratch arenas on demand, so their
// first call (and any call with larger sizes) runs cudaMalloc.  Some callers cannot allow that:
//  * a caller that sized the resident tensor to fill the device leaves no room for a later
//    cudaMalloc, which would fail with out-of-memory in the middle of an SCF;
//  * cudaFree (run when an arena grows) synchronises the whole device, which stalls work the
//    caller keeps in flight on its other streams;
//  * a host that owns the device memory through its own pool (a caching allocator, a Fortran or
//    Go driver with a fixed budget) does not want a library allocating beside it.
// rr_ri_coulomb_noalloc runs the same two TMA streaming passes as the Fock builds
// (gamma = B vec(D), then J = B^T gamma; reference src/NON_REL/NonRelFockMatrixRi.cpp:88-91) with all
// scratch in one fixed file-scope device array, and touches no allocator.
#include <mutex>

#include "j_stream.cuh"
#include "ri_store.cuh"

namespace rr {
namespace {

// 32 MiB of doubles.  Layout per call (each region 256-byte aligned):
//   [pitched copy of D: round_up(n^2, 32)] [J for host outputs: round_up(n^2, 32)]
//   [pass-1 partials: round_up(naux * nseg, 32)] [pass-2 partials: nrange * n^2]
// nrange (the aux ranges pass 2 splits over) shrinks to what fits; at least one must fit.
constexpr int64_t kScratchDoubles = 4LL << 20;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_scratch_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on `device` (which must be current).  The first call on a
// device looks it up with cudaGetSymbolAddress, which may load this module onto the device.
double* scratch_for(int device) {
  RR_REQUIRE(device >= 0 && device < kMaxDevices, RR_ERR_ARG, "rr_ri_coulomb_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      throw Error(RR_ERR_CUDA, std::string("rr_ri_coulomb_noalloc: cudaGetSymbolAddress failed: ") +
                                   cudaGetErrorString(e));
    g_scratch_ptr[device] = static_cast<double*>(p);
  }
  return g_scratch_ptr[device];
}

void coulomb_noalloc(rr_ri_store* h, const double* D, double* J, const rr_opts* o) {
  RR_REQUIRE(h->ntens == 1, RR_ERR_STATE, "rr_ri_coulomb_noalloc: handle holds a 4-component store");
  const bool host = !o || o->mem == RR_MEM_HOST;
  cudaStream_t s = call_stream(h, o);
  double* base = scratch_for(h->ctx.device);

  const int64_t n2 = h->n * h->n;
  const int64_t dpitch = round_up(std::max<int64_t>(n2, 2), 32);
  double* Dp = base;
  double* Jh = Dp + dpitch;
  const int64_t jh = host ? round_up(std::max<int64_t>(n2, 1), 32) : 0;

  JTensor t;
  t.B = h->B[0].p;
  t.pitch = h->pitch[0];
  t.len = n2;
  t.D = Dp;
  t.J = host ? Jh : J;
  JPlan pl = j_plan(1, &t, h->naux, 3);
  const int64_t gpart = round_up(std::max<int64_t>(pl.gpart_doubles, 1), 32);
  const int64_t fixed = dpitch + jh + gpart;
  const int64_t room = kScratchDoubles - fixed;
  if (n2 > 0 && room < n2) {
    throw Error(RR_ERR_ARG, "rr_ri_coulomb_noalloc: n = " + std::to_string(h->n) + ", naux = " +
                                std::to_string(h->naux) + " needs at least " + std::to_string(fixed + n2) +
                                " doubles of scratch; the fixed scratch holds " + std::to_string(kScratchDoubles) +
                                " (32 MiB); use rr_ri_jk_occupied or rr_ri_fock_nonrel for this size");
  }
  if (n2 > 0) {
    pl.nrange = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(pl.nrange, room / n2)));
    pl.jpart_doubles = static_cast<int64_t>(pl.nrange) * n2;
  }
  double* gp = Jh + jh;
  double* jp = gp + gpart;

  // The one padding entry past n^2 (odd n) is read by pass 1 against B's zero padding: it must be
  // finite, so it is cleared on every call.  All other regions are written before they are read.
  if (n2 > 0) {
    RR_CUDA(cudaMemcpyAsync(Dp, D, sizeof(double) * n2, host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
    if (dpitch > n2) RR_CUDA(cudaMemsetAsync(Dp + n2, 0, sizeof(double) * (dpitch - n2), s));
  }
  j_pass1(pl, gp, h->status.p, s);
  j_pass2(pl, gp, jp, h->status.p, s);
  j_finish(pl, jp, 1.0, s);
  if (host && n2 > 0) RR_CUDA(cudaMemcpyAsync(J, Jh, sizeof(double) * n2, cudaMemcpyDeviceToHost, s));
  if (host || (o && o->sync)) check_status(h, s);
}

}  // namespace
}  // namespace rr

extern "C" int rr_ri_coulomb_noalloc(rr_ri_handle h, const double* D, double* J, const rr_opts* opts) {
  try {
    rr::set_last_error("");
    if (!h) throw rr::Error(RR_ERR_ARG, "null handle");
    RR_REQUIRE(D && J, RR_ERR_ARG, "rr_ri_coulomb_noalloc: null matrix");
    RR_REQUIRE(!opts || opts->precision == RR_PREC_FP64, RR_ERR_UNSUPPORTED, "rr_ri_coulomb_noalloc: precision");
    RR_CUDA(cudaSetDevice(h->ctx.device));
    rr::coulomb_noalloc(h, D, J, opts);
    return RR_OK;
  } catch (const rr::Error& e) {
    rr::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    rr::set_last_error(e.what());
    return RR_ERR_CUDA;
  }
}
