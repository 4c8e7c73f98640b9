// Test hooks for the library's failure detection and allocation behaviour (declared in
// include/rr_ri_testing.h).  No reference counterpart.
#include <algorithm>

#include "ri_store.cuh"
#include "gemm_f64.cuh"
#include "tma_util.cuh"

namespace rr {
int64_t device_allocations();

namespace {

constexpr int kExpiryCode = 0x40;

// One CTA.  Thread 0 initialises an mbarrier that expects one arrival; nothing ever arrives and no
// bulk copy is issued, so every thread's bounded wait (the same mbar_wait the TMA pipelines use)
// polls `limit` times, records kExpiryCode in *err and returns false.  out[0]: SM cycles thread 0
// spent in the wait; out[1]: 1 if any wait returned true (it must not).
__global__ void wait_expiry_kernel(uint32_t limit, int* err, long long* out) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int completed;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
    completed = 0;
  }
  __syncthreads();
  const long long t0 = clock64();
  bool dead = false;
  const bool ok = mbar_wait(&bar, 0, err, kExpiryCode, dead, limit);
  const long long t1 = clock64();
  if (ok) atomicOr(&completed, 1);
  // a dead thread skips later waits at once: the second wait must return false without polling
  const bool again = mbar_wait(&bar, 0, err, kExpiryCode, dead, limit);
  if (again) atomicOr(&completed, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    out[0] = t1 - t0;
    out[1] = completed;
  }
}

// Status word of the half-transform hooks (per device, zeroed on first use): a timed-out wait of the
// bulk-copy pipeline sets it and the hook reports RR_ERR_TIMEOUT.
int* test_status() {
  static int* word[kMaxDevices] = {};
  const int d = current_device();
  if (!word[d]) {
    RR_CUDA(cudaMalloc(&word[d], sizeof(int)));
    RR_CUDA(cudaMemset(word[d], 0, sizeof(int)));
  }
  return word[d];
}

void check_test_status() {
  int v = 0;
  RR_CUDA(cudaMemcpy(&v, test_status(), sizeof(int), cudaMemcpyDeviceToHost));
  if (v) {
    RR_CUDA(cudaMemset(test_status(), 0, sizeof(int)));
    throw Error(RR_ERR_TIMEOUT, "half-transform pipeline wait timed out (status " + std::to_string(v) + ")");
  }
}

}  // namespace
}  // namespace rr

using rr::check_test_status;
using rr::test_status;

extern "C" {

int64_t rr_test_device_allocations(void) { return rr::device_allocations(); }

int rr_test_half_transform(const double* Ct, int64_t nocc, const double* B, int64_t naux, int64_t n, double* T,
                           int32_t variant) {
  try {
    rr::set_last_error("");
    RR_REQUIRE(variant >= 0 && variant <= 14, RR_ERR_ARG, "rr_test_half_transform: variant must be in [0, 14]");
    if (variant >= 1) {
      RR_REQUIRE(rr::half_transform_m16(Ct, nocc, B, n * n, naux, n, T, nullptr, variant - 1, test_status()),
                 RR_ERR_UNSUPPORTED,
                 "rr_test_half_transform: operands not supported by the m16n8k8 kernel");
    } else {
      rr::GemmDesc g;
      g.M = nocc; g.N = n; g.K = n;
      g.A = Ct; g.lda = n; g.strideA = 0;
      g.B = B; g.ldb = n; g.strideB = n * n;
      g.C = T; g.ldc = n; g.strideC = nocc * n;
      g.batch = naux;
      rr::gemm(g, nullptr);
    }
    RR_CUDA(cudaDeviceSynchronize());
    check_test_status();
    return RR_OK;
  } catch (const rr::Error& e) {
    rr::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    rr::set_last_error(e.what());
    return RR_ERR_CUDA;
  }
}

int rr_test_half_transform_time(const double* Ct, int64_t nocc, const double* B, int64_t naux, int64_t n, double* T,
                                int32_t variant, int32_t reps, double* ms) {
  try {
    rr::set_last_error("");
    RR_REQUIRE(reps >= 1 && ms, RR_ERR_ARG, "rr_test_half_transform_time: reps >= 1 and an output are needed");
    const int rc = rr_test_half_transform(Ct, nocc, B, naux, n, T, variant);  // warm-up, checks the variant
    if (rc != RR_OK) return rc;
    cudaEvent_t e0, e1;
    RR_CUDA(cudaEventCreate(&e0));
    RR_CUDA(cudaEventCreate(&e1));
    RR_CUDA(cudaEventRecord(e0, nullptr));
    for (int r = 0; r < reps; ++r) {
      if (variant >= 1) {
        rr::half_transform_m16(Ct, nocc, B, n * n, naux, n, T, nullptr, variant - 1, test_status());
      } else {
        rr::GemmDesc g;
        g.M = nocc; g.N = n; g.K = n;
        g.A = Ct; g.lda = n; g.B = B; g.ldb = n; g.strideB = n * n; g.C = T; g.ldc = n; g.strideC = nocc * n;
        g.batch = naux;
        rr::gemm(g, nullptr);
      }
    }
    RR_CUDA(cudaEventRecord(e1, nullptr));
    RR_CUDA(cudaEventSynchronize(e1));
    float t = 0.f;
    RR_CUDA(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check_test_status();
    *ms = t / reps;
    return RR_OK;
  } catch (const rr::Error& e) {
    rr::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    rr::set_last_error(e.what());
    return RR_ERR_CUDA;
  }
}

int rr_test_wait_expiry(uint32_t spin_limit, int32_t threads, int32_t* status_word, double* elapsed_ms,
                        double* cycles) {
  try {
    rr::set_last_error("");
    RR_REQUIRE(spin_limit >= 1 && spin_limit <= rr::kSpinLimit, RR_ERR_ARG,
               "rr_test_wait_expiry: spin_limit must be in [1, 4194304]");
    RR_REQUIRE(threads >= 32 && threads <= 1024 && threads % 32 == 0, RR_ERR_ARG,
               "rr_test_wait_expiry: threads must be a multiple of 32 in [32, 1024]");
    rr::DevBuf<int> err(1);
    rr::DevBuf<long long> out(2);
    RR_CUDA(cudaMemset(err.p, 0, sizeof(int)));
    RR_CUDA(cudaMemset(out.p, 0, 2 * sizeof(long long)));
    cudaEvent_t e0, e1;
    RR_CUDA(cudaEventCreate(&e0));
    RR_CUDA(cudaEventCreate(&e1));
    RR_CUDA(cudaEventRecord(e0, nullptr));
    rr::wait_expiry_kernel<<<1, threads>>>(spin_limit, err.p, out.p);
    RR_LAUNCH_CHECK();
    RR_CUDA(cudaEventRecord(e1, nullptr));
    RR_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    RR_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int word = 0;
    long long o[2] = {0, 0};
    RR_CUDA(cudaMemcpy(&word, err.p, sizeof(int), cudaMemcpyDeviceToHost));
    RR_CUDA(cudaMemcpy(o, out.p, sizeof(o), cudaMemcpyDeviceToHost));
    if (status_word) *status_word = word;
    if (elapsed_ms) *elapsed_ms = ms;
    if (cycles) *cycles = static_cast<double>(o[0]);
    RR_REQUIRE(o[1] == 0, RR_ERR_STATE, "rr_test_wait_expiry: a wait on a barrier nobody arrives on completed");
    // The pipelines report an expired wait as RR_ERR_TIMEOUT; so does this hook.
    if (word != 0) throw rr::Error(RR_ERR_TIMEOUT, "device wait bound expired (status word 0x" + std::to_string(word) + ")");
    return RR_OK;
  } catch (const rr::Error& e) {
    rr::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    rr::set_last_error(e.what());
    return RR_ERR_CUDA;
  }
}

}  // extern "C"
