// RESTART files (the reference's binary run-state format, src/Utils/Restart.h:14-70) and the device
// helpers that turn their coefficients into the next run's starting density, so that a chain of
// geometries (a scan) can hand its orbitals from one run to the next.
//
// The byte layout is the reference's, field for field (a file written here is read by the reference
// and the other way round): magic "RERDMFT\0", uint32 version 3, uint32 byte-order marker 0x01020304,
// three length-prefixed strings, the uint64 basis fingerprint, six int64 window counts, the double
// energy, two uint8 flags, three length-prefixed double vectors, the uint8 complex flag, uint64 rows
// and cols, the row-major coefficients, and the version-3 CASSCF section (two int64 and one vector).
// Version-2 files (no CASSCF section) are read too.
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "ri_store.cuh"

namespace rr {
namespace {

constexpr char kMagic[8] = {'R', 'E', 'R', 'D', 'M', 'F', 'T', '\0'};
constexpr uint32_t kVersion = 3;
constexpr uint32_t kOrderMark = 0x01020304u;
constexpr uint64_t kMaxCount = 1ULL << 40;  // bound on any count read from a file

bool little_endian() {
  const uint32_t v = kOrderMark;
  unsigned char b[4];
  std::memcpy(b, &v, 4);
  return b[0] == 0x04;
}

struct Writer {
  std::ofstream out;
  template <typename V>
  void put(V v) { out.write(reinterpret_cast<const char*>(&v), sizeof(V)); }
  void str(const char* s) {
    const std::string t = s ? s : "";
    put<uint64_t>(t.size());
    out.write(t.data(), static_cast<std::streamsize>(t.size()));
  }
  void vec(const double* p, int64_t n) {
    put<uint64_t>(static_cast<uint64_t>(n));
    if (n > 0) out.write(reinterpret_cast<const char*>(p), static_cast<std::streamsize>(n * sizeof(double)));
  }
};

struct Reader {
  std::ifstream in;
  template <typename V>
  V get() {
    V v{};
    in.read(reinterpret_cast<char*>(&v), sizeof(V));
    RR_REQUIRE(static_cast<bool>(in), RR_ERR_ARG, "readRestart: the file is truncated");
    return v;
  }
  char* str() {
    const auto n = get<uint64_t>();
    RR_REQUIRE(n <= 4096, RR_ERR_ARG, "readRestart: implausible string length");
    char* s = static_cast<char*>(std::calloc(n + 1, 1));
    RR_REQUIRE(s != nullptr, RR_ERR_NOMEM, "readRestart: host allocation failed");
    in.read(s, static_cast<std::streamsize>(n));
    RR_REQUIRE(static_cast<bool>(in), RR_ERR_ARG, "readRestart: the file is truncated");
    return s;
  }
  double* vec(int64_t* count) {
    const auto n = get<uint64_t>();
    RR_REQUIRE(n <= kMaxCount, RR_ERR_ARG, "readRestart: implausible vector length");
    *count = static_cast<int64_t>(n);
    return doubles(n);
  }
  double* doubles(uint64_t n) {
    double* p = static_cast<double*>(std::malloc(std::max<uint64_t>(n, 1) * sizeof(double)));
    RR_REQUIRE(p != nullptr, RR_ERR_NOMEM, "readRestart: host allocation failed");
    if (n > 0) in.read(reinterpret_cast<char*>(p), static_cast<std::streamsize>(n * sizeof(double)));
    RR_REQUIRE(static_cast<bool>(in), RR_ERR_ARG, "readRestart: the file is truncated");
    return p;
  }
};

bool str_is(const char* s, const char* v) { return s && std::strcmp(s, v) == 0; }

void write_restart(const char* path, const rr_restart* d) {
  RR_REQUIRE(path && d, RR_ERR_ARG, "writeRestart: null argument");
  RR_REQUIRE(little_endian(), RR_ERR_UNSUPPORTED, "writeRestart: big-endian hosts are not supported");
  RR_REQUIRE(str_is(d->kind, "OCCUPATIONS") || str_is(d->kind, "GAMMAS") || str_is(d->kind, "PCCD") ||
                 str_is(d->kind, "CASSCF"),
             RR_ERR_ARG, "writeRestart: kind must be OCCUPATIONS, GAMMAS, PCCD or CASSCF");
  RR_REQUIRE(!str_is(d->kind, "CASSCF") || (d->cas_electrons > 0 && d->cas_spinors > 0 && d->n_cas_state > 0),
             RR_ERR_ARG, "writeRestart: kind CASSCF without the active space or the CI vector");
  RR_REQUIRE(d->n_occupations > 0 && d->occupations, RR_ERR_ARG, "writeRestart: no occupation numbers");
  RR_REQUIRE(!str_is(d->kind, "GAMMAS") || d->n_gammas > 0, RR_ERR_ARG, "writeRestart: kind GAMMAS without gamma angles");
  RR_REQUIRE(!str_is(d->kind, "PCCD") || d->n_amplitudes > 0, RR_ERR_ARG,
             "writeRestart: kind PCCD without t-/z-amplitudes");
  RR_REQUIRE(d->rows > 0 && d->cols > 0 && d->coefficients, RR_ERR_ARG,
             "writeRestart: the coefficient matrix is missing or inconsistent");
  Writer w;
  w.out.open(path, std::ios::binary | std::ios::trunc);
  RR_REQUIRE(static_cast<bool>(w.out), RR_ERR_ARG, std::string("writeRestart: cannot open ") + path + " for writing");
  w.out.write(kMagic, sizeof(kMagic));
  w.put<uint32_t>(kVersion);
  w.put<uint32_t>(kOrderMark);
  w.str(d->method);
  w.str(d->functional);
  w.str(d->kind);
  w.put<uint64_t>(d->basis_fingerprint);
  for (int64_t v : {d->n_electrons, d->pnof_subspaces, d->pnof_coupling, d->n_core, d->jk_frozen_pairs,
                    d->jk_active_pairs})
    w.put<int64_t>(v);
  w.put<double>(d->total_energy);
  w.put<uint8_t>(d->orbitals_optimized ? 1 : 0);
  w.put<uint8_t>(d->converged ? 1 : 0);
  w.vec(d->occupations, d->n_occupations);
  w.vec(d->gammas, d->n_gammas);
  w.vec(d->amplitudes, d->n_amplitudes);
  w.put<uint8_t>(d->complex_coefficients ? 1 : 0);
  w.put<uint64_t>(static_cast<uint64_t>(d->rows));
  w.put<uint64_t>(static_cast<uint64_t>(d->cols));
  const int64_t entries = d->rows * d->cols * (d->complex_coefficients ? 2 : 1);
  w.out.write(reinterpret_cast<const char*>(d->coefficients), static_cast<std::streamsize>(entries * sizeof(double)));
  w.put<int64_t>(d->cas_electrons);
  w.put<int64_t>(d->cas_spinors);
  w.vec(d->cas_state, d->n_cas_state);
  w.out.flush();
  RR_REQUIRE(static_cast<bool>(w.out), RR_ERR_ARG, std::string("writeRestart: error while writing ") + path);
}

void release_restart(rr_restart* d) {
  if (!d) return;
  std::free(const_cast<char*>(d->method));
  std::free(const_cast<char*>(d->functional));
  std::free(const_cast<char*>(d->kind));
  std::free(const_cast<double*>(d->occupations));
  std::free(const_cast<double*>(d->gammas));
  std::free(const_cast<double*>(d->amplitudes));
  std::free(const_cast<double*>(d->coefficients));
  std::free(const_cast<double*>(d->cas_state));
  std::memset(d, 0, sizeof(*d));
}

void read_restart(const char* path, rr_restart* d) {
  RR_REQUIRE(path && d, RR_ERR_ARG, "readRestart: null argument");
  RR_REQUIRE(little_endian(), RR_ERR_UNSUPPORTED, "readRestart: big-endian hosts are not supported");
  std::memset(d, 0, sizeof(*d));
  Reader r;
  r.in.open(path, std::ios::binary);
  RR_REQUIRE(static_cast<bool>(r.in), RR_ERR_ARG, std::string("readRestart: cannot open ") + path);
  char magic[8];
  r.in.read(magic, sizeof(magic));
  RR_REQUIRE(static_cast<bool>(r.in) && std::memcmp(magic, kMagic, sizeof(kMagic)) == 0, RR_ERR_ARG,
             std::string("readRestart: ") + path + " is not a RERDMFT restart file");
  const auto version = r.get<uint32_t>();
  RR_REQUIRE(version == kVersion || version == 2, RR_ERR_ARG, "readRestart: unsupported restart-file version");
  RR_REQUIRE(r.get<uint32_t>() == kOrderMark, RR_ERR_ARG, "readRestart: the file has a different byte order");
  try {
    d->method = r.str();
    d->functional = r.str();
    d->kind = r.str();
    d->basis_fingerprint = r.get<uint64_t>();
    d->n_electrons = r.get<int64_t>();
    d->pnof_subspaces = r.get<int64_t>();
    d->pnof_coupling = r.get<int64_t>();
    d->n_core = r.get<int64_t>();
    d->jk_frozen_pairs = r.get<int64_t>();
    d->jk_active_pairs = r.get<int64_t>();
    d->total_energy = r.get<double>();
    d->orbitals_optimized = r.get<uint8_t>() != 0;
    d->converged = r.get<uint8_t>() != 0;
    d->occupations = r.vec(&d->n_occupations);
    d->gammas = r.vec(&d->n_gammas);
    d->amplitudes = r.vec(&d->n_amplitudes);
    d->complex_coefficients = r.get<uint8_t>() != 0;
    const auto rows = r.get<uint64_t>(), cols = r.get<uint64_t>();
    RR_REQUIRE(rows <= kMaxCount && cols <= kMaxCount && rows * cols <= kMaxCount, RR_ERR_ARG,
               "readRestart: implausible coefficient-matrix size");
    d->rows = static_cast<int64_t>(rows);
    d->cols = static_cast<int64_t>(cols);
    d->coefficients = r.doubles(rows * cols * (d->complex_coefficients ? 2 : 1));
    if (version >= 3) {
      d->cas_electrons = r.get<int64_t>();
      d->cas_spinors = r.get<int64_t>();
      d->cas_state = r.vec(&d->n_cas_state);
    }
  } catch (...) {
    release_restart(d);
    throw;
  }
}

// P = C diag(occ) C^dagger (rows x rows) for C rows x cols (real or interleaved complex).
__global__ void scale_columns_kernel(double* out, const double* C, const double* occ, int64_t rows, int64_t cols,
                                     int PL) {
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < rows * cols;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double o = occ[e % cols];
    out[PL * e] = C[PL * e] * o;
    if (PL == 2) out[2 * e + 1] = C[2 * e + 1] * o;
  }
}

}  // namespace
}  // namespace rr

namespace {
template <typename F>
int restart_api(F&& f) {
  try {
    rr::set_last_error("");
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
}  // namespace

extern "C" {

int rr_restart_write(const char* path, const rr_restart* data) {
  return restart_api([&] { rr::write_restart(path, data); });
}

int rr_restart_read(const char* path, rr_restart* out) {
  return restart_api([&] { rr::read_restart(path, out); });
}

int rr_restart_release(rr_restart* data) {
  return restart_api([&] { rr::release_restart(data); });
}

int rr_restart_coefficients(const double* c_scf, int64_t rows, int64_t n_mo, const double* u, int32_t cplx, double* c_out,
                            const rr_opts* opts) {
  return restart_api([&] {
    RR_REQUIRE(c_scf && c_out && rows >= 0 && n_mo >= 0, RR_ERR_ARG, "restartCoefficients: bad arguments");
    const int PL = cplx ? 2 : 1;
    const bool host = !opts || opts->mem == RR_MEM_HOST;
    const int64_t cn = rows * n_mo * PL;
    if (!u) {  // an empty rotation is the identity (src/Utils/Restart.cpp:199)
      if (c_out != c_scf && cn > 0)
        RR_CUDA(cudaMemcpy(c_out, c_scf, sizeof(double) * cn, host ? cudaMemcpyHostToHost : cudaMemcpyDeviceToDevice));
      return;
    }
    cudaStream_t s = opts && opts->stream ? static_cast<cudaStream_t>(opts->stream) : nullptr;
    rr::DevBuf<double> tc, tu, to;
    const double* cd = c_scf;
    const double* ud = u;
    double* od = c_out;
    if (host) {
      tc.alloc(static_cast<size_t>(std::max<int64_t>(cn, 1)));
      tu.alloc(static_cast<size_t>(std::max<int64_t>(n_mo * n_mo * PL, 1)));
      to.alloc(static_cast<size_t>(std::max<int64_t>(cn, 1)));
      RR_CUDA(cudaMemcpyAsync(tc.p, c_scf, sizeof(double) * cn, cudaMemcpyHostToDevice, s));
      RR_CUDA(cudaMemcpyAsync(tu.p, u, sizeof(double) * n_mo * n_mo * PL, cudaMemcpyHostToDevice, s));
      cd = tc.p;
      ud = tu.p;
      od = to.p;
    }
    rr::GemmDesc g;  // C = C_scf U
    g.cplx = cplx != 0;
    g.M = rows; g.N = n_mo; g.K = n_mo;
    g.A = cd; g.lda = n_mo; g.B = ud; g.ldb = n_mo; g.C = od; g.ldc = n_mo;
    rr::gemm(g, s);
    if (host) RR_CUDA(cudaMemcpyAsync(c_out, od, sizeof(double) * cn, cudaMemcpyDeviceToHost, s));
    RR_CUDA(cudaStreamSynchronize(s));
  });
}

int rr_density_from_orbitals(const double* C, int64_t rows, int64_t cols, const double* occupations, int32_t cplx,
                             double* P, const rr_opts* opts) {
  return restart_api([&] {
    RR_REQUIRE(C && occupations && P && rows >= 0 && cols >= 0, RR_ERR_ARG, "rr_density_from_orbitals: bad arguments");
    const int PL = cplx ? 2 : 1;
    const bool host = !opts || opts->mem == RR_MEM_HOST;
    cudaStream_t s = opts && opts->stream ? static_cast<cudaStream_t>(opts->stream) : nullptr;
    rr::DevBuf<double> tc, to, tp, sc(static_cast<size_t>(std::max<int64_t>(rows * cols * PL, 1)));
    const double* cd = C;
    const double* od = occupations;
    double* pd = P;
    if (host) {
      tc.alloc(static_cast<size_t>(std::max<int64_t>(rows * cols * PL, 1)));
      to.alloc(static_cast<size_t>(std::max<int64_t>(cols, 1)));
      tp.alloc(static_cast<size_t>(std::max<int64_t>(rows * rows * PL, 1)));
      RR_CUDA(cudaMemcpyAsync(tc.p, C, sizeof(double) * rows * cols * PL, cudaMemcpyHostToDevice, s));
      RR_CUDA(cudaMemcpyAsync(to.p, occupations, sizeof(double) * cols, cudaMemcpyHostToDevice, s));
      cd = tc.p;
      od = to.p;
      pd = tp.p;
    }
    if (rows > 0) {
      if (cols > 0) {
        rr::scale_columns_kernel<<<static_cast<int>(std::min<int64_t>(1184, (rows * cols + 255) / 256)), 256, 0, s>>>(
            sc.p, cd, od, rows, cols, PL);
        RR_LAUNCH_CHECK();
      }
      rr::GemmDesc g;  // P = (C diag(occ)) C^dagger, Hermitian: upper tiles and a mirror
      g.cplx = cplx != 0;
      g.M = rows; g.N = rows; g.K = cols;
      g.A = sc.p; g.lda = cols; g.B = cd; g.ldb = cols; g.opB = rr::Op::T; g.conjB = cplx != 0;
      g.C = pd; g.ldc = rows;
      g.mirror = 1;
      rr::gemm(g, s);
    }
    if (host) RR_CUDA(cudaMemcpyAsync(P, pd, sizeof(double) * rows * rows * PL, cudaMemcpyDeviceToHost, s));
    RR_CUDA(cudaStreamSynchronize(s));
  });
}

}  // extern "C"
