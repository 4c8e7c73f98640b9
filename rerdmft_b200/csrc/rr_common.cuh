// Shared runtime pieces of librr_ri: status codes, error capture, device buffers and the
// per-handle execution context (streams, events, cuSOLVER handle, scratch arena).
#pragma once

#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "rr_ri.h"

namespace rr {

// Error carried across the C ABI: every entry point catches rr::Error and returns its code.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

void set_last_error(const std::string& msg);

#define RR_CUDA(expr)                                                                          \
  do {                                                                                         \
    cudaError_t _e = (expr);                                                                   \
    if (_e != cudaSuccess)                                                                     \
      throw ::rr::Error(RR_ERR_CUDA, std::string(#expr " failed: ") + cudaGetErrorString(_e)); \
  } while (0)

#define RR_SOLVER(expr)                                                                          \
  do {                                                                                           \
    cusolverStatus_t _s = (expr);                                                                \
    if (_s != CUSOLVER_STATUS_SUCCESS)                                                           \
      throw ::rr::Error(RR_ERR_SOLVER, std::string(#expr " failed, status ") + std::to_string(_s)); \
  } while (0)

#define RR_REQUIRE(cond, code, msg)                \
  do {                                             \
    if (!(cond)) throw ::rr::Error((code), (msg)); \
  } while (0)

// Kernel launch check (configuration errors surface here; execution errors at the next sync);
// also counts the launch for rr_kernel_launches().
void count_launch();
#define RR_LAUNCH_CHECK()                                                                           \
  do {                                                                                              \
    cudaError_t _le = cudaGetLastError();                                                           \
    if (_le != cudaSuccess)                                                                         \
      throw ::rr::Error(RR_ERR_CUDA, std::string("kernel launch at " __FILE__ ":") +               \
                                         std::to_string(__LINE__) + ": " + cudaGetErrorString(_le)); \
    ::rr::count_launch();                                                                           \
  } while (0)

// Counts the device allocations the library makes (DevBuf::alloc); read by a test hook.
void count_device_alloc();

// Owning device allocation (cudaMalloc/cudaFree), move-only.
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  explicit DevBuf(size_t count) { alloc(count); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(size_t count) {
    release();
    if (count) {
      RR_CUDA(cudaMalloc(&p, count * sizeof(T)));
      count_device_alloc();
    }
    n = count;
  }
  // Grow-only: keeps the allocation when it is already large enough.
  void ensure(size_t count) { if (count > n) alloc(count); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// Execution context owned by a handle: a main stream (the caller's, or a private one), a side
// stream for the bandwidth-bound J pass that overlaps the exchange GEMMs, and fork/join events.
struct Context {
  int device = 0;
  cudaStream_t main = nullptr;
  cudaStream_t side = nullptr;
  bool own_main = false;
  cudaEvent_t fork = nullptr, join = nullptr, mid = nullptr;
  cudaEvent_t upl[3] = {nullptr, nullptr, nullptr};  // host-input uploads on the side stream
  // Second compute stream and its events: the exchange SYRK of one chunk of aux indices runs there
  // while the main stream half-transforms the next chunk.
  static constexpr int kPipeMax = 8;
  cudaStream_t pipe_stream = nullptr;
  cudaEvent_t pipe_ev[kPipeMax + 1] = {};
  cusolverDnHandle_t solver = nullptr;
  DevBuf<double> solver_work;
  DevBuf<int> solver_info;
  void init(cudaStream_t user_stream);
  void destroy();
  void set_stream(cudaStream_t s);
};

// CUDA keeps kernel attributes per device context.  One-time settings (dynamic shared-memory size,
// carveout) and the SM count are therefore kept per device ordinal, so one process may drive
// several GPUs (a handle binds to the device current at its creation).
constexpr int kMaxDevices = 64;
int current_device();
// Multiprocessor count of the current device (cached per device).
int sm_count_current();
// Runs f() once per device for this flag array (on the first call with that device current).
// Host threads may race into f() together for one device: the attributes it sets are idempotent.
template <class F>
void once_per_device(std::atomic<bool> (&done)[kMaxDevices], F&& f) {
  const int d = current_device();
  if (d < 0 || d >= kMaxDevices) {
    f();
    return;
  }
  if (!done[d].load(std::memory_order_acquire)) {
    f();
    done[d].store(true, std::memory_order_release);
  }
}

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }
inline int ceil_div(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

}  // namespace rr
