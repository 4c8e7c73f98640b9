// Store lifetime, streams, host<->device staging, small elementwise kernels and the FP64
// eigensolver wrapper shared by the Fock builds.
#include <algorithm>
#include <atomic>
#include <complex>

#include "ri_store.cuh"

namespace rr {

thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }

static std::atomic<int64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
int64_t launches() { return g_launches.load(std::memory_order_relaxed); }

static std::atomic<int64_t> g_device_allocs{0};
void count_device_alloc() { g_device_allocs.fetch_add(1, std::memory_order_relaxed); }
int64_t device_allocations() { return g_device_allocs.load(std::memory_order_relaxed); }

int current_device() {
  int dev = 0;
  RR_CUDA(cudaGetDevice(&dev));
  return dev;
}

int sm_count_current() {
  static std::atomic<int> cache[kMaxDevices];
  const int dev = current_device();
  int sms = (dev >= 0 && dev < kMaxDevices) ? cache[dev].load(std::memory_order_relaxed) : 0;
  if (sms > 0) return sms;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  if (dev >= 0 && dev < kMaxDevices) cache[dev].store(sms, std::memory_order_relaxed);
  return sms;
}

void Context::init(cudaStream_t user_stream) {
  RR_CUDA(cudaGetDevice(&device));
  if (user_stream) {
    main = user_stream;
    own_main = false;
  } else {
    RR_CUDA(cudaStreamCreateWithFlags(&main, cudaStreamNonBlocking));
    own_main = true;
  }
  // The side stream carries the bandwidth-bound Coulomb passes that run alongside compute-bound
  // GEMMs on the main stream; its higher priority lets their CTAs be dispatched as GEMM CTAs retire.
  int lo = 0, hi = 0;
  RR_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  RR_CUDA(cudaStreamCreateWithPriority(&side, cudaStreamNonBlocking, hi));
  RR_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  RR_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
  RR_CUDA(cudaEventCreateWithFlags(&mid, cudaEventDisableTiming));
  for (auto& e : upl) RR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  RR_CUDA(cudaStreamCreateWithFlags(&pipe_stream, cudaStreamNonBlocking));
  for (auto& e : pipe_ev) RR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  RR_SOLVER(cusolverDnCreate(&solver));
}

void Context::destroy() {
  if (solver) cusolverDnDestroy(solver);
  if (fork) cudaEventDestroy(fork);
  if (join) cudaEventDestroy(join);
  if (mid) cudaEventDestroy(mid);
  for (auto& e : upl) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  for (auto& e : pipe_ev) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  if (pipe_stream) cudaStreamDestroy(pipe_stream);
  pipe_stream = nullptr;
  if (side) cudaStreamDestroy(side);
  if (own_main && main) cudaStreamDestroy(main);
  solver = nullptr;
  fork = join = mid = nullptr;
  side = main = nullptr;
}

cudaStream_t call_stream(rr_ri_store* h, const rr_opts* o) {
  if (o && o->stream) return static_cast<cudaStream_t>(o->stream);
  return h->ctx.main;
}

void prof_mark(rr_ri_store* h, int i, cudaStream_t s) {
  if (!h->profiling) return;
  if (!h->ev[i]) RR_CUDA(cudaEventCreate(&h->ev[i]));
  RR_CUDA(cudaEventRecord(h->ev[i], s));
  h->ev_used[i] = true;
}

void host_wait(rr_ri_store* h, cudaStream_t s) {
  if (h && h->blocking_wait) {
    if (!h->wait_ev) RR_CUDA(cudaEventCreateWithFlags(&h->wait_ev, cudaEventBlockingSync | cudaEventDisableTiming));
    RR_CUDA(cudaEventRecord(h->wait_ev, s));
    RR_CUDA(cudaEventSynchronize(h->wait_ev));
  } else {
    RR_CUDA(cudaStreamSynchronize(s));
  }
}

void check_status(rr_ri_store* h, cudaStream_t s) {
  // word 0: bounded-wait expiries (TMA pipelines); word 1: numerical failures (recovery Cholesky)
  int word[2] = {0, 0};
  RR_CUDA(cudaMemcpyAsync(word, h->status.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  host_wait(h, s);
  if (word[0] != 0 || word[1] != 0) {
    RR_CUDA(cudaMemsetAsync(h->status.p, 0, 2 * sizeof(int), s));
    RR_CUDA(cudaStreamSynchronize(s));
    if (word[0] != 0)
      throw Error(RR_ERR_TIMEOUT, "device wait bound expired (status word 0x" + std::to_string(word[0]) + ")");
    throw Error(RR_ERR_SOLVER, "occupied recovery: the occupied-space Gram matrix is not positive definite");
  }
}

void copy_in(double* dst, const double* src, int64_t count, bool host, cudaStream_t s) {
  if (count <= 0) return;
  RR_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * count, host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
}

void copy_out(double* dst, const double* src, int64_t count, bool host, cudaStream_t s) {
  if (count <= 0) return;
  RR_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * count, host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s));
}

void copy_in_padded(double* dst, int64_t pitch, const double* src, int64_t n2, bool host, cudaStream_t s) {
  copy_in(dst, src, n2, host, s);
  if (pitch > n2) RR_CUDA(cudaMemsetAsync(dst + n2, 0, sizeof(double) * (pitch - n2), s));
}

namespace {

__global__ void axpby_kernel(double* y, const double* x, double a, double b, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    y[i] = a * x[i] + (b != 0.0 ? b * y[i] : 0.0);
}

__global__ void fock_combine_kernel(double* F, const double* h, const double* J, const double* K, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    F[i] = h[i] + J[i] - K[i];
}

__global__ void transpose_kernel(double* out, const double* in, int64_t rows, int64_t cols) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < rows * cols;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx / cols, j = idx % cols;
    out[j * rows + i] = in[idx];
  }
}

int blocks_for(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 1184))); }

}  // namespace

void axpby(double* y, const double* x, double a, double b, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  axpby_kernel<<<blocks_for(n), 256, 0, s>>>(y, x, a, b, n);
  RR_LAUNCH_CHECK();
}

void transpose(double* out, const double* in, int64_t rows, int64_t cols, cudaStream_t s) {
  if (rows * cols <= 0) return;
  transpose_kernel<<<blocks_for(rows * cols), 256, 0, s>>>(out, in, rows, cols);
  RR_LAUNCH_CHECK();
}

void fock_combine(double* F, const double* h, const double* J, const double* K, int64_t n2, cudaStream_t s) {
  if (n2 <= 0) return;
  fock_combine_kernel<<<blocks_for(n2), 256, 0, s>>>(F, h, J, K, n2);
  RR_LAUNCH_CHECK();
}

void eigh_sym_ctx(Context& c, double* a, int64_t n, double* w, cudaStream_t s) {
  if (n == 0) return;
  RR_SOLVER(cusolverDnSetStream(c.solver, s));
  int lwork = 0;
  RR_SOLVER(cusolverDnDsyevd_bufferSize(c.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, static_cast<int>(n),
                                        a, static_cast<int>(n), w, &lwork));
  c.solver_work.ensure(static_cast<size_t>(lwork) + 1);
  c.solver_info.ensure(1);
  RR_SOLVER(cusolverDnDsyevd(c.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, static_cast<int>(n), a,
                             static_cast<int>(n), w, c.solver_work.p, lwork, c.solver_info.p));
}

void eigh_herm_ctx(Context& c, double* a, int64_t n, double* w, cudaStream_t s) {
  if (n == 0) return;
  RR_SOLVER(cusolverDnSetStream(c.solver, s));
  int lwork = 0;
  auto* az = reinterpret_cast<cuDoubleComplex*>(a);
  RR_SOLVER(cusolverDnZheevd_bufferSize(c.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, static_cast<int>(n),
                                        az, static_cast<int>(n), w, &lwork));
  c.solver_work.ensure(2 * static_cast<size_t>(lwork) + 2);
  c.solver_info.ensure(1);
  RR_SOLVER(cusolverDnZheevd(c.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, static_cast<int>(n), az,
                             static_cast<int>(n), w, reinterpret_cast<cuDoubleComplex*>(c.solver_work.p), lwork,
                             c.solver_info.p));
}

void eigh_sym(rr_ri_store* h, double* a, int64_t n, double* w, cudaStream_t s) { eigh_sym_ctx(h->ctx, a, n, w, s); }

void eigh_herm(rr_ri_store* h, double* a, int64_t n, double* w, cudaStream_t s) { eigh_herm_ctx(h->ctx, a, n, w, s); }

}  // namespace rr
