// extern "C" boundary of librr_ri (declared in include/rr_ri.h).  Every entry point converts
// rr::Error (and any other exception) into a status code plus rr_last_error().
#include <algorithm>
#include <atomic>
#include <new>
#include <thread>
#include <vector>

#include "grouped.cuh"
#include "mo_store.cuh"

namespace rr {
extern thread_local std::string g_last_error;
void fock_nonrel(rr_ri_store*, const double*, const double*, const double*, const double*, int64_t, double*,
                 const rr_opts*);
void jk_occupied(rr_ri_store*, const double*, int64_t, double*, double*, const rr_opts*);
void fock_x2c(rr_ri_store*, const double*, const double*, const double*, const double*, int64_t, double*,
              const rr_opts*, const RelBuild* = nullptr, const double* = nullptr, int64_t = 0);
void ukb_two_electron(rr_ri_store*, const double*, const double*, int64_t, const double*, double*, const rr_opts*);
void fock_rkb(rr_ri_store*, const double*, const double*, int64_t, const double*, const double*, int64_t,
              const double*, double*, const rr_opts*, const RelBuild* = nullptr, const double* = nullptr,
              int64_t = 0);
void scf_nonrel(rr_ri_store*, const double*, const double*, int64_t, const double*, const double*, int,
                const rr_scf_opts*, rr_scf_result*, double*, double*, const rr_opts*);
void scf_x2c_grouped(rr_x2c_instance*, int64_t, const rr_scf_opts*, rr_batch_stats*);
void scf_rel(rr_ri_store*, int, const double*, const double*, int64_t, const double*, int64_t, const double*,
             const double*, int, const rr_scf_opts*, rr_scf_result*, double*, double*, const rr_opts*);
}  // namespace rr

namespace {

template <typename F>
int api(F&& f) {
  try {
    rr::g_last_error.clear();
    f();
    return RR_OK;
  } catch (const rr::Error& e) {
    rr::set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    rr::set_last_error("host allocation failed");
    return RR_ERR_NOMEM;
  } catch (const std::exception& e) {
    rr::set_last_error(e.what());
    return RR_ERR_CUDA;
  }
}

void upload_tensor(rr::DevBuf<double>& dst, int64_t* pitch_out, const double* src, int64_t naux, int64_t n2, bool host,
                   cudaStream_t s) {
  const int64_t pitch = rr::round_up(std::max<int64_t>(n2, 2), 32);
  *pitch_out = pitch;
  dst.alloc(static_cast<size_t>(std::max<int64_t>(naux * pitch, 32)));
  RR_CUDA(cudaMemsetAsync(dst.p, 0, sizeof(double) * dst.n, s));
  if (naux && n2)
    RR_CUDA(cudaMemcpy2DAsync(dst.p, sizeof(double) * pitch, src, sizeof(double) * n2, sizeof(double) * n2, naux,
                              host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
}

rr_mo_store* new_mo(int cplx, int64_t naux, int64_t n) {
  auto* m = new rr_mo_store();
  try {
    m->ctx.init(nullptr);
  } catch (...) {
    delete m;
    throw;
  }
  m->cplx = cplx;
  m->naux = naux;
  m->n = n;
  return m;
}

void free_mo(rr_mo_store* m) {
  if (!m) return;
  m->ctx.destroy();
  delete m;
}

rr_mo_store* checked_mo(rr_mo_handle m) {
  if (!m) throw rr::Error(RR_ERR_ARG, "null MO handle");
  RR_CUDA(cudaSetDevice(m->ctx.device));
  return m;
}

bool host_mem(const rr_opts* o) { return !o || o->mem == RR_MEM_HOST; }

template <typename F>
void with_new_mo(rr_mo_handle* out, rr_mo_store* m, F&& f) {
  try {
    f();
  } catch (...) {
    free_mo(m);
    throw;
  }
  *out = m;
}


// Clears an SCF result record for a new run, keeping the output pointers the caller set in it.
void keep_outputs_reset(rr_scf_result* r) {
  double* w = r->orbital_energies;
  double* c = r->c_matrix;
  double* f = r->fock_matrix;
  *r = rr_scf_result{};
  r->orbital_energies = w;
  r->c_matrix = c;
  r->fock_matrix = f;
}

rr_ri_store* checked(rr_ri_handle h) {
  if (!h) throw rr::Error(RR_ERR_ARG, "null handle");
  RR_CUDA(cudaSetDevice(h->ctx.device));
  return h;
}

}  // namespace

extern "C" {

const char* rr_last_error(void) { return rr::g_last_error.c_str(); }

int rr_version(void) { return 100; }

int rr_ri_create(const double* B, int64_t naux, int64_t n, int32_t mem, rr_ri_handle* out) {
  return api([&] {
    RR_REQUIRE(out != nullptr, RR_ERR_ARG, "rr_ri_create: out is null");
    *out = nullptr;
    RR_REQUIRE(naux >= 0 && n >= 1, RR_ERR_ARG, "rr_ri_create: need naux >= 0 and n >= 1");
    RR_REQUIRE(B != nullptr || naux == 0, RR_ERR_ARG, "rr_ri_create: B is null");
    RR_REQUIRE(mem == RR_MEM_HOST || mem == RR_MEM_DEVICE, RR_ERR_ARG, "rr_ri_create: bad mem kind");
    auto* h = new rr_ri_store();
    try {
      h->ctx.init(nullptr);
      h->naux = naux;
      h->n = n;
      h->ntens = 1;
      h->status.alloc(2);
      RR_CUDA(cudaMemsetAsync(h->status.p, 0, 2 * sizeof(int), h->ctx.main));
      upload_tensor(h->B[0], &h->pitch[0], B, naux, n * n, mem == RR_MEM_HOST, h->ctx.main);
      rr::pack_for_j(h, 0, n, h->ctx.main);
      RR_CUDA(cudaStreamSynchronize(h->ctx.main));
    } catch (...) {
      h->ctx.destroy();
      delete h;
      throw;
    }
    *out = h;
  });
}

int rr_ri_create_4c(const double* B_LL, const double* B_SS, int64_t naux, int64_t nl, int64_t ns, int32_t mem,
                    rr_ri_handle* out) {
  return api([&] {
    RR_REQUIRE(out != nullptr, RR_ERR_ARG, "rr_ri_create_4c: out is null");
    *out = nullptr;
    RR_REQUIRE(naux >= 0 && nl >= 1 && ns >= 0, RR_ERR_ARG, "rr_ri_create_4c: bad dimensions");
    RR_REQUIRE((B_LL && (B_SS || ns == 0)) || naux == 0, RR_ERR_ARG, "rr_ri_create_4c: null tensor");
    RR_REQUIRE(mem == RR_MEM_HOST || mem == RR_MEM_DEVICE, RR_ERR_ARG, "rr_ri_create_4c: bad mem kind");
    auto* h = new rr_ri_store();
    try {
      h->ctx.init(nullptr);
      h->naux = naux;
      h->n = nl;
      h->ns = ns;
      h->ntens = 2;
      h->status.alloc(2);
      RR_CUDA(cudaMemsetAsync(h->status.p, 0, 2 * sizeof(int), h->ctx.main));
      upload_tensor(h->B[0], &h->pitch[0], B_LL, naux, nl * nl, mem == RR_MEM_HOST, h->ctx.main);
      upload_tensor(h->B[1], &h->pitch[1], B_SS, naux, ns * ns, mem == RR_MEM_HOST, h->ctx.main);
      rr::pack_for_j(h, 0, nl, h->ctx.main);
      rr::pack_for_j(h, 1, ns, h->ctx.main);
      RR_CUDA(cudaStreamSynchronize(h->ctx.main));
    } catch (...) {
      h->ctx.destroy();
      delete h;
      throw;
    }
    *out = h;
  });
}

int rr_ri_destroy(rr_ri_handle h) {
  return api([&] {
    if (!h) return;
    cudaSetDevice(h->ctx.device);
    cudaDeviceSynchronize();
    for (auto& e : h->ev)
      if (e) cudaEventDestroy(e);
    if (h->wait_ev) cudaEventDestroy(h->wait_ev);
    h->ctx.destroy();
    delete h;
  });
}

int rr_ri_info(rr_ri_handle h, int64_t* naux, int64_t* n, int64_t* ns) {
  return api([&] {
    if (!h) throw rr::Error(RR_ERR_ARG, "null handle");
    if (naux) *naux = h->naux;
    if (n) *n = h->n;
    if (ns) *ns = h->ns;
  });
}

int rr_ri_sync(rr_ri_handle h) {
  return api([&] {
    auto* s = checked(h);
    RR_CUDA(cudaStreamSynchronize(s->ctx.side));
    rr::check_status(s, s->ctx.main);
  });
}

int rr_ri_fock_nonrel(rr_ri_handle h, const double* h_core, const double* D, const double* S, const double* X,
                      int64_t n_eff, double* F, const rr_opts* opts) {
  return api([&] {
    auto* s = checked(h);
    RR_REQUIRE(h_core && D && S && F && (X || n_eff == 0), RR_ERR_ARG, "rr_ri_fock_nonrel: null matrix");
    RR_REQUIRE(!opts || opts->precision == RR_PREC_FP64, RR_ERR_UNSUPPORTED,
               "rr_ri_fock_nonrel: only RR_PREC_FP64 (the mixed path runs through rr_ri_jk_occupied / the SCF driver)");
    rr::fock_nonrel(s, h_core, D, S, X, n_eff, F, opts);
  });
}

int rr_ri_jk_occupied(rr_ri_handle h, const double* C_occ, int64_t n_occ, double* J, double* K, const rr_opts* opts) {
  return api([&] {
    auto* s = checked(h);
    RR_REQUIRE((C_occ || n_occ == 0) && J && K, RR_ERR_ARG, "rr_ri_jk_occupied: null matrix");
    RR_REQUIRE(!opts || opts->precision == RR_PREC_FP64 || opts->precision == RR_PREC_MIXED, RR_ERR_UNSUPPORTED,
               "rr_ri_jk_occupied: unknown precision");
    rr::jk_occupied(s, C_occ, n_occ, J, K, opts);
  });
}

int rr_ri_fock_x2c(rr_ri_handle h, const double* h_x2c, const double* P, const double* S, const double* X,
                   int64_t n_eff, double* F, const rr_opts* opts) {
  return api([&] {
    auto* s = checked(h);
    RR_REQUIRE(h_x2c && P && S && F && (X || n_eff == 0), RR_ERR_ARG, "rr_ri_fock_x2c: null matrix");
    RR_REQUIRE(!opts || opts->precision == RR_PREC_FP64 || opts->precision == RR_PREC_MIXED, RR_ERR_UNSUPPORTED,
               "rr_ri_fock_x2c: precision");
    rr::RelBuild rb;
    rb.mixed = true;
    rb.incremental = opts && opts->incremental != 0;
    rr::fock_x2c(s, h_x2c, P, S, X, n_eff, F, opts, opts && opts->precision == RR_PREC_MIXED ? &rb : nullptr);
  });
}

int rr_ri_two_electron_ukb(rr_ri_handle h, const double* P_ukb, const double* C_occ, int64_t n_occ,
                           const double* occupations, double* G, const rr_opts* opts) {
  return api([&] {
    auto* s = checked(h);
    RR_REQUIRE(P_ukb && G && ((C_occ && occupations) || n_occ == 0), RR_ERR_ARG, "rr_ri_two_electron_ukb: null matrix");
    RR_REQUIRE(!opts || opts->precision == RR_PREC_FP64, RR_ERR_UNSUPPORTED, "rr_ri_two_electron_ukb: precision");
    rr::ukb_two_electron(s, P_ukb, C_occ, n_occ, occupations, G, opts);
  });
}

int rr_ri_fock_rkb(rr_ri_handle h, const double* h_rkb, const double* v_total, int64_t n_rkb, const double* s_full,
                   const double* x_full, int64_t n_eff, const double* P, double* F, const rr_opts* opts) {
  return api([&] {
    auto* s = checked(h);
    RR_REQUIRE(h_rkb && v_total && s_full && P && F && (x_full || n_eff == 0), RR_ERR_ARG, "rr_ri_fock_rkb: null matrix");
    RR_REQUIRE(!opts || opts->precision == RR_PREC_FP64 || opts->precision == RR_PREC_MIXED, RR_ERR_UNSUPPORTED,
               "rr_ri_fock_rkb: precision");
    rr::RelBuild rb;
    rb.mixed = true;
    rb.incremental = opts && opts->incremental != 0;
    rr::fock_rkb(s, h_rkb, v_total, n_rkb, s_full, x_full, n_eff, P, F, opts,
                 opts && opts->precision == RR_PREC_MIXED ? &rb : nullptr);
  });
}

int rr_scf_run_nonrel(rr_ri_handle h, const double* h_core, const double* X, int64_t n_eff, const double* S,
                      const double* P0, int32_t n_electrons, const rr_scf_opts* scf, rr_scf_result* result,
                      double* P_out, double* energy_history, const rr_opts* opts) {
  return api([&] {
    auto* s = checked(h);
    RR_REQUIRE(h_core && X && S && P0 && scf && result && P_out, RR_ERR_ARG, "rr_scf_run_nonrel: null argument");
    RR_REQUIRE(n_eff >= 1 && n_eff <= s->n, RR_ERR_ARG, "rr_scf_run_nonrel: n_eff out of range");
    RR_REQUIRE(scf->max_iterations >= 1, RR_ERR_ARG, "rr_scf_run_nonrel: max_iterations < 1");
    RR_REQUIRE(scf->precision == RR_PREC_FP64 || scf->precision == RR_PREC_MIXED, RR_ERR_UNSUPPORTED,
               "rr_scf_run_nonrel: unknown precision");
    keep_outputs_reset(result);
    rr::scf_nonrel(s, h_core, X, n_eff, S, P0, n_electrons, scf, result, P_out, energy_history, opts);
  });
}

int rr_scf_run_x2c(rr_ri_handle h, const double* h_x2c, const double* X, int64_t n_eff, const double* S,
                   const double* P0, int32_t n_electrons, const rr_scf_opts* scf, rr_scf_result* result,
                   double* P_out, double* energy_history, const rr_opts* opts) {
  return api([&] {
    auto* s = checked(h);
    RR_REQUIRE(s->ntens == 1, RR_ERR_STATE, "rr_scf_run_x2c: handle holds a 4-component store");
    RR_REQUIRE(h_x2c && X && S && P0 && scf && result && P_out, RR_ERR_ARG, "rr_scf_run_x2c: null argument");
    RR_REQUIRE(n_eff >= 1 && n_eff <= 2 * s->n, RR_ERR_ARG, "rr_scf_run_x2c: n_eff out of range");
    RR_REQUIRE(scf->max_iterations >= 1, RR_ERR_ARG, "rr_scf_run_x2c: max_iterations < 1");
    RR_REQUIRE(scf->precision == RR_PREC_FP64 || scf->precision == RR_PREC_MIXED, RR_ERR_UNSUPPORTED,
               "rr_scf_run_x2c: precision");
    keep_outputs_reset(result);
    rr::scf_rel(s, 0, h_x2c, nullptr, 2 * s->n, X, n_eff, S, P0, n_electrons, scf, result, P_out, energy_history,
                opts);
  });
}

int rr_scf_run_x2c_grouped(rr_x2c_instance* instances, int64_t count, const rr_scf_opts* scf, rr_batch_stats* stats) {
  return api([&] {
    RR_REQUIRE(count >= 0 && (instances || count == 0) && scf, RR_ERR_ARG, "rr_scf_run_x2c_grouped: null argument");
    if (stats) *stats = rr_batch_stats{};
    if (count == 0) return;
    RR_CUDA(cudaSetDevice(instances[0].h ? instances[0].h->ctx.device : 0));
    for (int64_t i = 0; i < count; ++i)
      RR_REQUIRE(!instances[i].h || instances[i].h->ctx.device == instances[0].h->ctx.device, RR_ERR_ARG,
                 "rr_scf_run_x2c_grouped: every handle must live on one device");
    rr::scf_x2c_grouped(instances, count, scf, stats);
    for (int64_t i = 0; i < count; ++i)
      if (instances[i].status != RR_OK)
        throw rr::Error(instances[i].status, "rr_scf_run_x2c_grouped: instance " + std::to_string(i) + " failed");
  });
}

int rr_autotune_load(const char* path) {
  return api([&] {
    RR_REQUIRE(path, RR_ERR_ARG, "rr_autotune_load: null path");
    rr::autotune_load(path);
  });
}

int rr_autotune_save(const char* path) {
  return api([&] {
    RR_REQUIRE(path, RR_ERR_ARG, "rr_autotune_save: null path");
    rr::autotune_save(path);
  });
}

int rr_autotune_clear(void) {
  return api([&] { rr::autotune_clear(); });
}

int64_t rr_autotune_entries(void) { return rr::autotune_entries(); }

int rr_scf_run_x2c_batch(rr_x2c_instance* instances, int64_t count, const rr_scf_opts* scf, int32_t workers) {
  return api([&] {
    RR_REQUIRE(count >= 0 && (instances || count == 0) && scf, RR_ERR_ARG, "rr_scf_run_x2c_batch: null argument");
    RR_REQUIRE(workers >= 1, RR_ERR_ARG, "rr_scf_run_x2c_batch: workers < 1");
    // Largest first (by the store's naux * n^2, which sets the cost of a build), so that no large
    // instance starts last and leaves the other workers idle.
    std::vector<int64_t> order(static_cast<size_t>(count));
    std::vector<double> cost(static_cast<size_t>(count), 0.0);
    for (int64_t i = 0; i < count; ++i) {
      order[i] = i;
      if (instances[i].h) {
        const rr_ri_store* st = instances[i].h;
        cost[i] = static_cast<double>(st->naux) * static_cast<double>(st->n) * static_cast<double>(st->n);
      }
    }
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return cost[a] > cost[b]; });
    std::atomic<int64_t> next{0};
    auto work = [&] {
      for (;;) {
        const int64_t k = next.fetch_add(1);
        if (k >= count) return;
        rr_x2c_instance& in = instances[order[k]];
        in.status = rr_scf_run_x2c(in.h, in.h_x2c, in.X, in.n_eff, in.S, in.P0, in.n_electrons, scf, &in.result,
                                   in.P_out, in.energy_history, nullptr);
      }
    };
    const int nw = static_cast<int>(std::min<int64_t>(workers, std::max<int64_t>(count, 1)));
    // With several workers the SCF host waits sleep instead of spinning (the threads would otherwise
    // compete for the host cores while their GPU work runs); restored afterwards.
    std::vector<char> was(static_cast<size_t>(count), 0);
    for (int64_t i = 0; i < count; ++i)
      if (instances[i].h) {
        was[i] = instances[i].h->blocking_wait ? 1 : 0;
        instances[i].h->blocking_wait = nw > 1;
      }
    std::vector<std::thread> pool;
    for (int w = 1; w < nw; ++w) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    for (int64_t i = 0; i < count; ++i)
      if (instances[i].h) instances[i].h->blocking_wait = was[i] != 0;
    for (int64_t i = 0; i < count; ++i)
      if (instances[i].status != RR_OK)
        throw rr::Error(instances[i].status, "rr_scf_run_x2c_batch: instance " + std::to_string(i) + " failed");
  });
}

int rr_scf_run_dhf(rr_ri_handle h, const double* h_rkb, const double* v_total, int64_t n_rkb, const double* s_full,
                   const double* x_full, const double* P0, int32_t n_electrons, const rr_scf_opts* scf,
                   rr_scf_result* result, double* P_out, double* energy_history, const rr_opts* opts) {
  return api([&] {
    auto* s = checked(h);
    RR_REQUIRE(s->ntens == 2, RR_ERR_STATE, "rr_scf_run_dhf: needs a 4-component store (rr_ri_create_4c)");
    RR_REQUIRE(h_rkb && v_total && s_full && x_full && P0 && scf && result && P_out, RR_ERR_ARG,
               "rr_scf_run_dhf: null argument");
    RR_REQUIRE(n_rkb >= 4 && n_rkb % 4 == 0, RR_ERR_ARG,
               "rkbDensityMatrix: RKB basis dimension must be even (4*nLarge)");
    RR_REQUIRE(scf->max_iterations >= 1, RR_ERR_ARG, "rr_scf_run_dhf: max_iterations < 1");
    RR_REQUIRE(scf->precision == RR_PREC_FP64 || scf->precision == RR_PREC_MIXED, RR_ERR_UNSUPPORTED,
               "rr_scf_run_dhf: precision");
    keep_outputs_reset(result);
    rr::scf_rel(s, 1, h_rkb, v_total, n_rkb, x_full, n_rkb, s_full, P0, n_electrons, scf, result, P_out,
                energy_history, opts);
  });
}

int rr_ri_set_profiling(rr_ri_handle h, int32_t on) {
  return api([&] {
    auto* s = checked(h);
    s->profiling = on != 0;
    for (bool& u : s->ev_used) u = false;
  });
}

int rr_ri_get_timings(rr_ri_handle h, rr_timings* out) {
  return api([&] {
    auto* s = checked(h);
    RR_REQUIRE(out != nullptr, RR_ERR_ARG, "rr_ri_get_timings: out is null");
    *out = rr_timings{};
    RR_REQUIRE(s->ev_used[0] && s->ev_used[4], RR_ERR_STATE, "rr_ri_get_timings: no profiled call recorded");
    RR_CUDA(cudaEventSynchronize(s->ev[4]));
    auto el = [&](int a, int b) -> double {
      if (!s->ev_used[a] || !s->ev_used[b]) return 0.0;
      float ms = 0.f;
      RR_CUDA(cudaEventSynchronize(s->ev[b]));
      RR_CUDA(cudaEventElapsedTime(&ms, s->ev[a], s->ev[b]));
      return static_cast<double>(ms);
    };
    out->total_ms = el(0, 4);
    out->recovery_ms = el(0, 1);
    out->half_transform_ms = el(1, 2);
    out->exchange_ms = s->ev_used[2] ? el(2, 3) : el(1, 3);
    out->coulomb_ms = el(5, 6);
    out->epilogue_ms = el(3, 4);
  });
}

int64_t rr_kernel_launches(void) { return rr::launches(); }

// ---------------- MO tensors ----------------

int rr_mo_build_nonrel(rr_ri_handle ri, const double* C, rr_mo_handle* out, const rr_opts* opts) {
  return api([&] {
    auto* s = checked(ri);
    RR_REQUIRE(out && C, RR_ERR_ARG, "rr_mo_build_nonrel: null argument");
    *out = nullptr;
    RR_REQUIRE(s->ntens == 1, RR_ERR_STATE, "rr_mo_build_nonrel: needs a single-tensor handle");
    auto* m = new_mo(0, s->naux, s->n);
    with_new_mo(out, m, [&] {
      cudaStream_t st = rr::call_stream(s, opts);
      if (opts && opts->precision == RR_PREC_MIXED) {
        rr::mo_build_nonrel_mixed(s, C, m, host_mem(opts), st);
        rr::check_status(s, st);
      } else {
        rr::mo_build_nonrel(s, C, m, host_mem(opts), st);
      }
      RR_CUDA(cudaStreamSynchronize(st));
    });
  });
}

int rr_mo_build_nonrel_into(rr_ri_handle ri, const double* C, rr_mo_handle mo, const rr_opts* opts) {
  return api([&] {
    auto* s = checked(ri);
    RR_REQUIRE(C, RR_ERR_ARG, "rr_mo_build_nonrel_into: null argument");
    auto* m = checked_mo(mo);
    RR_REQUIRE(s->ntens == 1, RR_ERR_STATE, "rr_mo_build_nonrel_into: needs a single-tensor handle");
    RR_REQUIRE(!m->cplx && m->naux == s->naux && m->n == s->n, RR_ERR_ARG,
               "rr_mo_build_nonrel_into: the MO handle is not a nonrelativistic tensor of the handle's naux and n");
    cudaStream_t st = rr::call_stream(s, opts);
    const bool mixed = opts && opts->precision == RR_PREC_MIXED;
    if (mixed) rr::mo_build_nonrel_mixed(s, C, m, host_mem(opts), st);
    else rr::mo_build_nonrel(s, C, m, host_mem(opts), st);
    if (host_mem(opts) || (opts && opts->sync)) {
      if (mixed) rr::check_status(s, st);
      RR_CUDA(cudaStreamSynchronize(st));
    }
  });
}

int rr_mo_build_ukb(rr_ri_handle ri4c, const double* c_ukb, int64_t n_total, rr_mo_handle* out, const rr_opts* opts) {
  return api([&] {
    auto* s = checked(ri4c);
    RR_REQUIRE(out && (c_ukb || n_total == 0) && n_total >= 0, RR_ERR_ARG, "rr_mo_build_ukb: bad argument");
    *out = nullptr;
    RR_REQUIRE(s->ntens == 2, RR_ERR_STATE, "rr_mo_build_ukb: needs a 4-component handle (rr_ri_create_4c)");
    auto* m = new_mo(1, s->naux, n_total);
    with_new_mo(out, m, [&] {
      cudaStream_t st = rr::call_stream(s, opts);
      if (opts && opts->precision == RR_PREC_MIXED) {
        rr::mo_build_ukb_mixed(s, c_ukb, n_total, m, host_mem(opts), st);
        rr::check_status(s, st);
      } else {
        rr::mo_build_ukb(s, c_ukb, n_total, m, host_mem(opts), st);
      }
      RR_CUDA(cudaStreamSynchronize(st));
    });
  });
}

int rr_mo_hx_joint_hessian_diagonal(rr_mo_handle mh, const double* h, const double* occupations,
                                    const double* two_rdm_h, const double* two_rdm_x, const double* fock,
                                    int64_t n_pairs, const int64_t* pairs, const int64_t* pair_of,
                                    const double* two_rdm_l1, const double* two_rdm_l2, double* out,
                                    const rr_opts* opts) {
  return api([&] {
    auto* m = checked_mo(mh);
    RR_REQUIRE(h && occupations && two_rdm_h && two_rdm_x && fock && out && n_pairs >= 0 && (pairs || n_pairs == 0),
               RR_ERR_ARG, "hartreeExchangeJointHessianDiagonal: null argument");
    RR_REQUIRE(!pair_of || (two_rdm_l1 && two_rdm_l2), RR_ERR_ARG,
               "hartreeExchangeJointHessianDiagonal: pair_of/two_rdm_l1/two_rdm_l2 must be given together");
    cudaStream_t st = rr::mo_stream(m, opts);
    rr::mo_hx_joint_hessian_diagonal(m, h, occupations, two_rdm_h, two_rdm_x, fock, n_pairs, pairs, pair_of,
                                     two_rdm_l1, two_rdm_l2, out, host_mem(opts), st);
    if (host_mem(opts) || (opts && opts->sync)) RR_CUDA(cudaStreamSynchronize(st));
  });
}

int rr_mo_cas_two_electron(rr_mo_handle mh, const double* rho, double* G, const rr_opts* opts) {
  return api([&] {
    auto* m = checked_mo(mh);
    RR_REQUIRE(rho && G, RR_ERR_ARG, "casTwoElectronOperator: null matrix");
    cudaStream_t st = rr::mo_stream(m, opts);
    rr::cas_two_electron(m, rho, G, host_mem(opts), st);
    if (host_mem(opts) || (opts && opts->sync)) RR_CUDA(cudaStreamSynchronize(st));
  });
}

int rr_mo_cas_cumulant_fock(rr_mo_handle mh, int64_t n_active, const int64_t* active, const double* lambda, double* F,
                            const rr_opts* opts) {
  return api([&] {
    auto* m = checked_mo(mh);
    RR_REQUIRE(n_active >= 0 && (n_active == 0 || (active && lambda)) && F, RR_ERR_ARG,
               "casActiveCumulantFock: bad arguments");
    cudaStream_t st = rr::mo_stream(m, opts);
    rr::cas_cumulant_fock(m, n_active, active, lambda, F, host_mem(opts), st);
    if (host_mem(opts) || (opts && opts->sync)) RR_CUDA(cudaStreamSynchronize(st));
  });
}

int rr_mo_cas_active_integrals(rr_mo_handle mh, int64_t n_active, const int64_t* active, double* out,
                               const rr_opts* opts) {
  return api([&] {
    auto* m = checked_mo(mh);
    RR_REQUIRE(n_active >= 0 && (n_active == 0 || (active && out)), RR_ERR_ARG, "casActiveIntegrals: bad arguments");
    cudaStream_t st = rr::mo_stream(m, opts);
    rr::cas_active_integrals(m, n_active, active, out, host_mem(opts), st);
    if (host_mem(opts) || (opts && opts->sync)) RR_CUDA(cudaStreamSynchronize(st));
  });
}

int rr_mo_from_tensor(const double* Bmo, int64_t naux, int64_t n, int32_t kind, int32_t mem, rr_mo_handle* out) {
  return api([&] {
    RR_REQUIRE(out && naux >= 0 && n >= 0 && (Bmo || naux * n == 0), RR_ERR_ARG, "rr_mo_from_tensor: bad argument");
    RR_REQUIRE(kind == RR_MO_NONREL_SPIN || kind == RR_MO_COMPLEX, RR_ERR_ARG, "rr_mo_from_tensor: bad kind");
    *out = nullptr;
    auto* m = new_mo(kind == RR_MO_COMPLEX, naux, n);
    with_new_mo(out, m, [&] {
      const int64_t cnt = naux * n * n * (kind == RR_MO_COMPLEX ? 2 : 1);
      m->B.alloc(static_cast<size_t>(std::max<int64_t>(cnt, 1)));
      rr::copy_in(m->B.p, Bmo, cnt, mem == RR_MEM_HOST, m->ctx.main);
      RR_CUDA(cudaStreamSynchronize(m->ctx.main));
    });
  });
}

int rr_mo_destroy(rr_mo_handle m) {
  return api([&] {
    if (!m) return;
    cudaSetDevice(m->ctx.device);
    cudaDeviceSynchronize();
    free_mo(m);
  });
}

int rr_mo_info(rr_mo_handle m, int64_t* naux, int64_t* n, int32_t* kind) {
  return api([&] {
    if (!m) throw rr::Error(RR_ERR_ARG, "null MO handle");
    if (naux) *naux = m->naux;
    if (n) *n = m->n;
    if (kind) *kind = m->cplx ? RR_MO_COMPLEX : RR_MO_NONREL_SPIN;
  });
}

int rr_mo_copy_tensor(rr_mo_handle m, double* out, const rr_opts* opts) {
  return api([&] {
    auto* s = checked_mo(m);
    RR_REQUIRE(out || s->naux * s->n == 0, RR_ERR_ARG, "rr_mo_copy_tensor: null output");
    cudaStream_t st = rr::mo_stream(s, opts);
    rr::copy_out(out, s->B.p, s->naux * s->n * s->n * (s->cplx ? 2 : 1), host_mem(opts), st);
    RR_CUDA(cudaStreamSynchronize(st));
  });
}

int rr_mo_rotated(rr_mo_handle m, const double* U, rr_mo_handle* out, const rr_opts* opts) {
  return api([&] {
    auto* s = checked_mo(m);
    RR_REQUIRE(out && U, RR_ERR_ARG, "rr_mo_rotated: null argument");
    *out = nullptr;
    auto* d = new_mo(s->cplx, s->naux, s->n);
    with_new_mo(out, d, [&] {
      cudaStream_t st = rr::mo_stream(s, opts);
      rr::mo_rotate(s, U, d, host_mem(opts), st);
      RR_CUDA(cudaStreamSynchronize(st));
    });
  });
}

int rr_mo_positive_block(rr_mo_handle m, int64_t off, rr_mo_handle* out, const rr_opts* opts) {
  return api([&] {
    auto* s = checked_mo(m);
    RR_REQUIRE(out && off >= 0 && off <= s->n, RR_ERR_ARG, "rr_mo_positive_block: bad offset");
    *out = nullptr;
    auto* d = new_mo(s->cplx, s->naux, s->n - off);
    with_new_mo(out, d, [&] {
      cudaStream_t st = rr::mo_stream(s, opts);
      rr::mo_positive_block(s, off, d, st);
      RR_CUDA(cudaStreamSynchronize(st));
    });
  });
}

int rr_mo_embedded(rr_mo_handle m, double* out, const rr_opts* opts) {
  return api([&] {
    auto* s = checked_mo(m);
    RR_REQUIRE(!s->cplx, RR_ERR_STATE, "rr_mo_embedded: only for the nonrelativistic spin-orbital kind");
    RR_REQUIRE(out || s->naux * s->n == 0, RR_ERR_ARG, "rr_mo_embedded: null output");
    cudaStream_t st = rr::mo_stream(s, opts);
    rr::mo_embedded(s, out, host_mem(opts), st);
    RR_CUDA(cudaStreamSynchronize(st));
  });
}

int rr_mo_eri(rr_mo_handle m, int64_t count, const int64_t* abcd, double* out, const rr_opts* opts) {
  return api([&] {
    auto* s = checked_mo(m);
    RR_REQUIRE(count >= 0 && (count == 0 || (abcd && out)), RR_ERR_ARG, "rr_mo_eri: bad argument");
    if (host_mem(opts)) {
      const int64_t dim = s->cplx ? s->n : 2 * s->n;
      for (int64_t i = 0; i < 4 * count; ++i)
        RR_REQUIRE(abcd[i] >= 0 && abcd[i] < dim, RR_ERR_ARG, "rr_mo_eri: index out of range");
    }
    cudaStream_t st = rr::mo_stream(s, opts);
    rr::mo_eri(s, count, abcd, out, host_mem(opts), st);
    RR_CUDA(cudaStreamSynchronize(st));
  });
}

int rr_mo_jkl(rr_mo_handle m, const int64_t* pair_of, double* J, double* K, double* L, const rr_opts* opts) {
  return api([&] {
    auto* s = checked_mo(m);
    RR_REQUIRE(J && K, RR_ERR_ARG, "rr_mo_jkl: null output");
    RR_REQUIRE(!L || pair_of, RR_ERR_ARG, "rr_mo_jkl: L needs pair_of");
    if (pair_of && host_mem(opts)) {
      const int64_t dim = s->cplx ? s->n : 2 * s->n;
      for (int64_t i = 0; i < dim; ++i)
        RR_REQUIRE(pair_of[i] >= 0 && pair_of[i] < dim, RR_ERR_ARG, "rr_mo_jkl: pair_of out of range");
    }
    cudaStream_t st = rr::mo_stream(s, opts);
    rr::mo_jkl(s, pair_of, J, K, L, host_mem(opts), st);
    RR_CUDA(cudaStreamSynchronize(st));
  });
}

int rr_mo_hx_fock(rr_mo_handle m, const double* h, const double* occupations, const double* two_rdm_h,
                  const double* two_rdm_x, const int64_t* pair_of, const double* two_rdm_l1, const double* two_rdm_l2,
                  double* F, const rr_opts* opts) {
  return api([&] {
    auto* s = checked_mo(m);
    RR_REQUIRE(h && occupations && two_rdm_h && two_rdm_x && F, RR_ERR_ARG, "rr_mo_hx_fock: null matrix");
    RR_REQUIRE(!pair_of || (two_rdm_l1 && two_rdm_l2), RR_ERR_ARG,
               "hartreeExchangeFockMatrix: pair_of/two_rdm_l1/two_rdm_l2 dimensions inconsistent with h");
    if (pair_of && host_mem(opts)) {
      const int64_t dim = s->cplx ? s->n : 2 * s->n;
      for (int64_t i = 0; i < dim; ++i)
        RR_REQUIRE(pair_of[i] >= 0 && pair_of[i] < dim, RR_ERR_ARG, "rr_mo_hx_fock: pair_of out of range");
    }
    cudaStream_t st = rr::mo_stream(s, opts);
    rr::mo_hx_fock(s, h, occupations, two_rdm_h, two_rdm_x, pair_of, two_rdm_l1, two_rdm_l2, F, host_mem(opts), st);
    RR_CUDA(cudaStreamSynchronize(st));
  });
}

}  // extern "C"

// ---- test hooks (include/rr_ri_testing.h) ----
extern "C" int rr_test_gemm_f64(int64_t M, int64_t N, int64_t K, const double* A, int64_t lda, int64_t strideA,
                                int32_t opA, const double* B, int64_t ldb, int64_t strideB, int32_t opB, double* C,
                                int64_t ldc, int64_t strideC, double alpha, double beta, int64_t batch, int32_t cplx,
                                int32_t conjA, int32_t conjB, int32_t mirror, int32_t allow_split) {
  return api([&] {
    rr::GemmDesc g;
    g.M = M; g.N = N; g.K = K;
    g.A = A; g.lda = lda; g.strideA = strideA; g.opA = opA ? rr::Op::T : rr::Op::N;
    g.B = B; g.ldb = ldb; g.strideB = strideB; g.opB = opB ? rr::Op::T : rr::Op::N;
    g.C = C; g.ldc = ldc; g.strideC = strideC;
    g.alpha = alpha; g.beta = beta; g.batch = batch;
    g.cplx = cplx != 0; g.conjA = conjA != 0; g.conjB = conjB != 0; g.mirror = mirror;
    rr::DevBuf<double> work;
    int64_t cap = 0;
    if (allow_split) {
      cap = rr::gemm_work_doubles(g);
      work.alloc(static_cast<size_t>(std::max<int64_t>(cap, 1)));
    }
    rr::gemm(g, nullptr, allow_split ? work.p : nullptr, cap);
    RR_CUDA(cudaDeviceSynchronize());
  });
}

extern "C" int rr_test_mixed_exchange(const double* B, int64_t naux, int64_t n, const double* Ct, int64_t nocc,
                                      double* K) {
  return api([&] {
    rr::MixedOperands mo;
    rr::MixedScratch scr;
    rr::DevBuf<int> err(2);
    RR_CUDA(cudaMemset(err.p, 0, 2 * sizeof(int)));
    rr::mixed_prepare(mo, B, n * n, n, naux, nullptr);
    rr::mixed_exchange(mo, scr, Ct, n, nocc, K, err.p, nullptr);
    RR_CUDA(cudaDeviceSynchronize());
    int e = 0;
    RR_CUDA(cudaMemcpy(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost));
    RR_REQUIRE(e == 0, RR_ERR_TIMEOUT, "rr_test_mixed_exchange: device wait bound expired (0x" + std::to_string(e) + ")");
  });
}

extern "C" int rr_test_mixed_exchange_delta(const double* B, int64_t naux, int64_t n, const double* Ct,
                                            const double* Ct_prev, int64_t nocc, double* dK) {
  return api([&] {
    rr::MixedOperands mo;
    rr::MixedScratch scr;
    rr::DevBuf<int> err(2);
    RR_CUDA(cudaMemset(err.p, 0, 2 * sizeof(int)));
    rr::mixed_prepare(mo, B, n * n, n, naux, nullptr);
    rr::ExFlavours fl;
    fl.nf = 1;
    fl.fs[0] = n;
    rr::mixed_exchange_general(&mo, scr, fl, naux, Ct, Ct_prev, n, nocc, false, dK, n, false, err.p, nullptr);
    RR_CUDA(cudaDeviceSynchronize());
    int e = 0;
    RR_CUDA(cudaMemcpy(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost));
    RR_REQUIRE(e == 0, RR_ERR_TIMEOUT,
               "rr_test_mixed_exchange_delta: device wait bound expired (0x" + std::to_string(e) + ")");
  });
}

extern "C" int rr_test_j_passes(const double* B, int64_t naux, int64_t n2, const double* D, double* gamma, double* J) {
  return api([&] {
    const int64_t pitch = rr::round_up(std::max<int64_t>(n2, 2), 32);
    rr::DevBuf<double> Bp(static_cast<size_t>(std::max<int64_t>(naux * pitch, 32))), Dp(static_cast<size_t>(pitch));
    rr::DevBuf<int> err(1);
    RR_CUDA(cudaMemset(Bp.p, 0, sizeof(double) * Bp.n));
    RR_CUDA(cudaMemset(Dp.p, 0, sizeof(double) * Dp.n));
    RR_CUDA(cudaMemset(err.p, 0, sizeof(int)));
    if (naux) RR_CUDA(cudaMemcpy2D(Bp.p, sizeof(double) * pitch, B, sizeof(double) * n2, sizeof(double) * n2, naux,
                                   cudaMemcpyDeviceToDevice));
    RR_CUDA(cudaMemcpy(Dp.p, D, sizeof(double) * n2, cudaMemcpyDeviceToDevice));
    rr::JTensor t;
    t.B = Bp.p; t.pitch = pitch; t.len = n2; t.D = Dp.p; t.J = J;
    rr::JPlan pl = rr::j_plan(1, &t, naux);
    rr::DevBuf<double> gp(static_cast<size_t>(std::max<int64_t>(pl.gpart_doubles, 1)));
    rr::DevBuf<double> jp(static_cast<size_t>(std::max<int64_t>(pl.jpart_doubles, 1)));
    rr::j_pass1(pl, gp.p, err.p, nullptr);
    rr::j_gamma(pl, gp.p, gamma, nullptr);
    rr::j_pass2(pl, gp.p, jp.p, err.p, nullptr);
    rr::j_finish(pl, jp.p, 1.0, nullptr);
    RR_CUDA(cudaDeviceSynchronize());
    int e = 0;
    RR_CUDA(cudaMemcpy(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost));
    RR_REQUIRE(e == 0, RR_ERR_TIMEOUT, "rr_test_j_passes: device wait bound expired");
  });
}

extern "C" int rr_test_j_passes_packed(const double* B, int64_t naux, int64_t n, const double* D, double* gamma,
                                       double* J, int32_t* packed) {
  return api([&] {
    RR_REQUIRE(naux >= 1 && n >= 1 && packed != nullptr, RR_ERR_ARG, "rr_test_j_passes_packed: bad arguments");
    const int64_t n2 = n * n;
    const int64_t pitch = rr::round_up(std::max<int64_t>(n2, 2), 32);
    rr::DevBuf<double> Bp(static_cast<size_t>(naux * pitch)), Bpk, Dpk(static_cast<size_t>(rr::tri_len(n) + 1));
    rr::DevBuf<double> Dp(static_cast<size_t>(pitch));  // zero-padded copy for the dense passes
    rr::DevBuf<int> err(1);
    RR_CUDA(cudaMemset(Bp.p, 0, sizeof(double) * Bp.n));
    RR_CUDA(cudaMemset(Dp.p, 0, sizeof(double) * Dp.n));
    RR_CUDA(cudaMemcpy(Dp.p, D, sizeof(double) * n2, cudaMemcpyDeviceToDevice));
    RR_CUDA(cudaMemset(err.p, 0, sizeof(int)));
    RR_CUDA(cudaMemcpy2D(Bp.p, sizeof(double) * pitch, B, sizeof(double) * n2, sizeof(double) * n2, naux,
                         cudaMemcpyDeviceToDevice));
    int64_t pitch_pk = 0;
    const bool ok = rr::j_pack_upper(Bp.p, pitch, naux, n, Bpk, pitch_pk, nullptr);
    *packed = ok ? 1 : 0;
    rr::JTensor t;
    t.J = J;
    if (ok) {
      rr::j_fold_density(D, n, Dpk.p, nullptr);
      t.B = Bpk.p; t.pitch = pitch_pk; t.len = rr::tri_len(n); t.tri_n = n; t.D = Dpk.p;
    } else {
      t.B = Bp.p; t.pitch = pitch; t.len = n2; t.D = Dp.p;
    }
    rr::JPlan pl = rr::j_plan(1, &t, naux);
    rr::DevBuf<double> gp(static_cast<size_t>(std::max<int64_t>(pl.gpart_doubles, 1)));
    rr::DevBuf<double> jp(static_cast<size_t>(std::max<int64_t>(pl.jpart_doubles, 1)));
    rr::j_pass1(pl, gp.p, err.p, nullptr);
    rr::j_gamma(pl, gp.p, gamma, nullptr);
    rr::j_pass2(pl, gp.p, jp.p, err.p, nullptr);
    rr::j_finish(pl, jp.p, 1.0, nullptr);
    RR_CUDA(cudaDeviceSynchronize());
    int e = 0;
    RR_CUDA(cudaMemcpy(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost));
    RR_REQUIRE(e == 0, RR_ERR_TIMEOUT, "rr_test_j_passes_packed: device wait bound expired");
  });
}
