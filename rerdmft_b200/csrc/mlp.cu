// The learned orbital-rotation preconditioner: an 8 -> 64 -> 64 -> 64 -> 1 multilayer perceptron
// (tanh hidden units, linear output) that predicts log |H_pp,qq| (the diagonal orbital Hessian of
// the functional stage) from eight per-pair inputs.  No counterpart in the reference: it rescales
// the ADAM pairs of the orbital optimisation, whose plain form stays the fallback.
//
// Training is FP32 on the GPU with these kernels only: a thread-per-sample forward pass that keeps
// the activations (feature-major, coalesced), a thread-per-sample backward pass for the deltas, a
// thread-per-parameter reduction over the batch for the weight gradients (fixed order, no atomics:
// identical results run to run), and Adam on the parameters.  Inference runs in BF16 (weights and
// activations rounded to bfloat16, FP32 accumulation).  Inputs and labels are standardised with the
// mean and spread of the first training set.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "rr_common.cuh"

namespace rr {
namespace {

constexpr int IN = 8, HID = 64;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + HID * IN, OFF_W2 = OFF_B1 + HID, OFF_B2 = OFF_W2 + HID * HID,
              OFF_W3 = OFF_B2 + HID, OFF_B3 = OFF_W3 + HID * HID, OFF_W4 = OFF_B3 + HID, OFF_B4 = OFF_W4 + HID,
              NPARAM = OFF_B4 + 1;  // 8961
constexpr int NNORM = 2 * IN + 2;  // x mean, x spread, y mean, y spread
constexpr int TPB = 128;

static_assert(NPARAM == 8961, "parameter layout");

__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// One hidden layer for one sample: out[j] = tanh(b[j] + sum_k W[j][k] in[k]) (W row-major HID x K).
template <int K, bool BF16>
__device__ __forceinline__ void dense_tanh(const float* W, const float* b, const float* in, float* out) {
#pragma unroll 4
  for (int j = 0; j < HID; ++j) {
    float acc = b[j];
#pragma unroll
    for (int k = 0; k < K; ++k) acc = fmaf(W[j * K + k], in[k], acc);
    const float t = tanhf(acc);
    out[j] = BF16 ? bf(t) : t;
  }
}

// Forward pass, thread per sample.  Xraw: count x 8 (host layout); rows idx[s] when idx != null.
// STORE keeps Xn (8 x count), A1..A3 (64 x count each) for the backward pass.
template <bool STORE, bool BF16>
__global__ void __launch_bounds__(TPB) mlp_forward_kernel(const float* params, const float* norm, const float* Xraw,
                                                          const int64_t* idx, int64_t count, float* Xn, float* A1,
                                                          float* A2, float* A3, float* yhat) {
  __shared__ float P[NPARAM];
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) P[i] = BF16 ? bf(params[i]) : params[i];
  __syncthreads();
  const int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (s >= count) return;
  const int64_t row = idx ? idx[s] : s;
  float x[IN], a[HID], c[HID];
#pragma unroll
  for (int k = 0; k < IN; ++k) {
    x[k] = (Xraw[row * IN + k] - norm[k]) / norm[IN + k];
    if (BF16) x[k] = bf(x[k]);
    if (STORE) Xn[k * count + s] = x[k];
  }
  dense_tanh<IN, BF16>(P + OFF_W1, P + OFF_B1, x, a);
  if (STORE)
    for (int j = 0; j < HID; ++j) A1[j * count + s] = a[j];
  dense_tanh<HID, BF16>(P + OFF_W2, P + OFF_B2, a, c);
  if (STORE)
    for (int j = 0; j < HID; ++j) A2[j * count + s] = c[j];
  dense_tanh<HID, BF16>(P + OFF_W3, P + OFF_B3, c, a);
  if (STORE)
    for (int j = 0; j < HID; ++j) A3[j * count + s] = a[j];
  float y = P[OFF_B4];
  for (int k = 0; k < HID; ++k) y = fmaf(P[OFF_W4 + k], a[k], y);
  yhat[s] = y;  // standardised units
}

// Backward pass, thread per sample: e = yhat - y_std, loss term e^2, delta4 = 2 e / count and the
// hidden deltas D3, D2, D1 (64 x count each).
__global__ void __launch_bounds__(TPB) mlp_backward_kernel(const float* params, const float* norm, const float* yraw,
                                                           const int64_t* idx, int64_t count, const float* A1,
                                                           const float* A2, const float* A3, const float* yhat,
                                                           float* D1, float* D2, float* D3, float* d4, float* err2) {
  __shared__ float P[NPARAM];
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) P[i] = params[i];
  __syncthreads();
  const int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (s >= count) return;
  const int64_t row = idx ? idx[s] : s;
  const float yt = (yraw[row] - norm[2 * IN]) / norm[2 * IN + 1];
  const float e = yhat[s] - yt;
  err2[s] = e * e;
  const float g4 = 2.0f * e / static_cast<float>(count);
  d4[s] = g4;
  float dl[HID], dn[HID];
  for (int k = 0; k < HID; ++k) {
    const float a = A3[k * count + s];
    dl[k] = P[OFF_W4 + k] * g4 * (1.0f - a * a);
    D3[k * count + s] = dl[k];
  }
  for (int k = 0; k < HID; ++k) {
    float acc = 0.0f;
    for (int j = 0; j < HID; ++j) acc = fmaf(P[OFF_W3 + j * HID + k], dl[j], acc);
    const float a = A2[k * count + s];
    dn[k] = acc * (1.0f - a * a);
    D2[k * count + s] = dn[k];
  }
  for (int k = 0; k < HID; ++k) {
    float acc = 0.0f;
    for (int j = 0; j < HID; ++j) acc = fmaf(P[OFF_W2 + j * HID + k], dn[j], acc);
    const float a = A1[k * count + s];
    D1[k * count + s] = acc * (1.0f - a * a);
  }
}

// Weight gradients, thread per parameter: dW_l[j][k] = sum_s D_l[j][s] in_l[k][s], db_l[j] =
// sum_s D_l[j][s], in order of s (deterministic).
__global__ void mlp_wgrad_kernel(const float* Xn, const float* A1, const float* A2, const float* A3, const float* D1,
                                 const float* D2, const float* D3, const float* d4, int64_t count, float* grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NPARAM) return;
  const float *D, *X;
  int off;
  if (i < OFF_B1) { D = D1 + ((i - OFF_W1) / IN) * count; X = Xn + ((i - OFF_W1) % IN) * count; off = 0; }
  else if (i < OFF_W2) { D = D1 + (i - OFF_B1) * count; X = nullptr; off = 1; }
  else if (i < OFF_B2) { D = D2 + ((i - OFF_W2) / HID) * count; X = A1 + ((i - OFF_W2) % HID) * count; off = 0; }
  else if (i < OFF_W3) { D = D2 + (i - OFF_B2) * count; X = nullptr; off = 1; }
  else if (i < OFF_B3) { D = D3 + ((i - OFF_W3) / HID) * count; X = A2 + ((i - OFF_W3) % HID) * count; off = 0; }
  else if (i < OFF_W4) { D = D3 + (i - OFF_B3) * count; X = nullptr; off = 1; }
  else if (i < OFF_B4) { D = d4; X = A3 + (i - OFF_W4) * count; off = 0; }
  else { D = d4; X = nullptr; off = 1; }
  float acc = 0.0f;
  if (off) {
    for (int64_t s = 0; s < count; ++s) acc += D[s];
  } else {
    for (int64_t s = 0; s < count; ++s) acc = fmaf(D[s], X[s], acc);
  }
  grad[i] = acc;
}

// out[0] = sum of `count` floats (one CTA, fixed order per thread then tree)
__global__ void sum_kernel(const float* v, int64_t count, float* out) {
  __shared__ float red[32];
  float a = 0.0f;
  for (int64_t i = threadIdx.x; i < count; i += blockDim.x) a += v[i];
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += red[w];
    out[0] = t;
  }
}

// Adam on the parameters (beta1 0.9, beta2 0.999, eps 1e-8).
__global__ void adam_f32_kernel(float* p, const float* g, float* m, float* v, int n, float lr, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = 0.9f * m[i] + 0.1f * gi;
  const float vi = 0.999f * v[i] + 0.001f * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
}

uint64_t splitmix(uint64_t& st) {
  uint64_t z = (st += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

double uniform01(uint64_t& st) { return static_cast<double>(splitmix(st) >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace
}  // namespace rr

struct rr_mlp_store {
  int device = 0;
  cudaStream_t s = nullptr;
  rr::DevBuf<float> params, norm, m, v, grad;
  std::vector<float> host_norm;
  bool has_norm = false;
  int64_t adam_t = 0;
  // training scratch
  rr::DevBuf<float> X, y, act, yhat, err2, scal;
  rr::DevBuf<int64_t> idx;
  int64_t cap = 0;

  void ensure_scratch(int64_t count, int64_t batch) {
    X.ensure(static_cast<size_t>(std::max<int64_t>(count * rr::IN, 1)));
    y.ensure(static_cast<size_t>(std::max<int64_t>(count, 1)));
    idx.ensure(static_cast<size_t>(std::max<int64_t>(count, 1)));
    if (batch > cap) {
      // Xn (8) + A1..A3 (3 x 64) + D1..D3 (3 x 64) + d4 (1) per sample
      act.alloc(static_cast<size_t>(batch * (rr::IN + 6 * rr::HID + 1)));
      yhat.alloc(static_cast<size_t>(batch));
      err2.alloc(static_cast<size_t>(batch));
      cap = batch;
    }
    scal.ensure(4);
  }
  // forward + backward + weight gradients over `count` samples (rows idx, or 0..count-1)
  void fwd_bwd(const float* Xd, const float* yd, const int64_t* id, int64_t count) {
    float* Xn = act.p;
    float* A1 = Xn + rr::IN * count;
    float* A2 = A1 + rr::HID * count;
    float* A3 = A2 + rr::HID * count;
    float* D1 = A3 + rr::HID * count;
    float* D2 = D1 + rr::HID * count;
    float* D3 = D2 + rr::HID * count;
    float* d4 = D3 + rr::HID * count;
    const int blocks = static_cast<int>((count + rr::TPB - 1) / rr::TPB);
    rr::mlp_forward_kernel<true, false><<<blocks, rr::TPB, 0, s>>>(params.p, norm.p, Xd, id, count, Xn, A1, A2, A3,
                                                                   yhat.p);
    RR_LAUNCH_CHECK();
    rr::mlp_backward_kernel<<<blocks, rr::TPB, 0, s>>>(params.p, norm.p, yd, id, count, A1, A2, A3, yhat.p, D1, D2,
                                                       D3, d4, err2.p);
    RR_LAUNCH_CHECK();
    rr::mlp_wgrad_kernel<<<(rr::NPARAM + 255) / 256, 256, 0, s>>>(Xn, A1, A2, A3, D1, D2, D3, d4, count, grad.p);
    RR_LAUNCH_CHECK();
    rr::sum_kernel<<<1, 256, 0, s>>>(err2.p, count, scal.p);
    RR_LAUNCH_CHECK();
  }
  void set_norm_from(const float* X, const float* yv, int64_t count) {
    host_norm.assign(rr::NNORM, 0.0f);
    for (int k = 0; k < rr::IN; ++k) {
      double mu = 0.0, sq = 0.0;
      for (int64_t i = 0; i < count; ++i) mu += X[i * rr::IN + k];
      mu /= static_cast<double>(count);
      for (int64_t i = 0; i < count; ++i) sq += (X[i * rr::IN + k] - mu) * (X[i * rr::IN + k] - mu);
      const double sd = std::sqrt(sq / static_cast<double>(count));
      host_norm[k] = static_cast<float>(mu);
      host_norm[rr::IN + k] = static_cast<float>(sd > 1e-12 ? sd : 1.0);
    }
    double mu = 0.0, sq = 0.0;
    for (int64_t i = 0; i < count; ++i) mu += yv[i];
    mu /= static_cast<double>(count);
    for (int64_t i = 0; i < count; ++i) sq += (yv[i] - mu) * (yv[i] - mu);
    const double sd = std::sqrt(sq / static_cast<double>(count));
    host_norm[2 * rr::IN] = static_cast<float>(mu);
    host_norm[2 * rr::IN + 1] = static_cast<float>(sd > 1e-12 ? sd : 1.0);
    RR_CUDA(cudaMemcpy(norm.p, host_norm.data(), sizeof(float) * rr::NNORM, cudaMemcpyHostToDevice));
    has_norm = true;
  }
};

namespace {

template <typename Fn>
int mlp_guard(Fn&& f) {
  try {
    rr::set_last_error("");
    f();
    return RR_OK;
  } catch (const rr::Error& e) {
    rr::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    rr::set_last_error(e.what());
    return RR_ERR_CUDA;
  }
}

rr_mlp_store* checked_mlp(rr_mlp_handle h) {
  if (!h) throw rr::Error(RR_ERR_ARG, "null MLP handle");
  RR_CUDA(cudaSetDevice(h->device));
  return h;
}

}  // namespace

extern "C" {

int rr_mlp_create(uint64_t seed, rr_mlp_handle* out) {
  return mlp_guard([&] {
    RR_REQUIRE(out, RR_ERR_ARG, "rr_mlp_create: null output");
    *out = nullptr;
    auto* h = new rr_mlp_store();
    try {
      RR_CUDA(cudaGetDevice(&h->device));
      RR_CUDA(cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking));
      h->params.alloc(rr::NPARAM);
      h->m.alloc(rr::NPARAM);
      h->v.alloc(rr::NPARAM);
      h->grad.alloc(rr::NPARAM);
      h->norm.alloc(rr::NNORM);
      // Xavier-uniform weights, zero biases (splitmix64 stream from the seed)
      std::vector<float> p(rr::NPARAM, 0.0f);
      uint64_t st = seed;
      auto fill = [&](int off, int fan_out, int fan_in) {
        const double lim = std::sqrt(6.0 / (fan_in + fan_out));
        for (int i = 0; i < fan_out * fan_in; ++i) p[off + i] = static_cast<float>((2.0 * rr::uniform01(st) - 1.0) * lim);
      };
      fill(rr::OFF_W1, rr::HID, rr::IN);
      fill(rr::OFF_W2, rr::HID, rr::HID);
      fill(rr::OFF_W3, rr::HID, rr::HID);
      fill(rr::OFF_W4, 1, rr::HID);
      RR_CUDA(cudaMemcpy(h->params.p, p.data(), sizeof(float) * rr::NPARAM, cudaMemcpyHostToDevice));
      RR_CUDA(cudaMemset(h->m.p, 0, sizeof(float) * rr::NPARAM));
      RR_CUDA(cudaMemset(h->v.p, 0, sizeof(float) * rr::NPARAM));
      std::vector<float> nm(rr::NNORM, 0.0f);
      for (int k = 0; k < rr::IN; ++k) nm[rr::IN + k] = 1.0f;
      nm[2 * rr::IN + 1] = 1.0f;
      h->host_norm = nm;
      RR_CUDA(cudaMemcpy(h->norm.p, nm.data(), sizeof(float) * rr::NNORM, cudaMemcpyHostToDevice));
    } catch (...) {
      if (h->s) cudaStreamDestroy(h->s);
      delete h;
      throw;
    }
    *out = h;
  });
}

int rr_mlp_destroy(rr_mlp_handle h) {
  return mlp_guard([&] {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->s) cudaStreamDestroy(h->s);
    delete h;
  });
}

int rr_mlp_train(rr_mlp_handle h, const float* X, const float* y, int64_t count, int32_t epochs, int32_t batch,
                 float learning_rate, uint64_t shuffle_seed, float* loss_per_epoch) {
  return mlp_guard([&] {
    auto* m = checked_mlp(h);
    RR_REQUIRE(X && y && count > 0 && epochs >= 0 && batch > 0, RR_ERR_ARG, "rr_mlp_train: bad arguments");
    if (!m->has_norm) m->set_norm_from(X, y, count);
    const int64_t bsz = std::min<int64_t>(batch, count);
    m->ensure_scratch(count, bsz);
    RR_CUDA(cudaMemcpyAsync(m->X.p, X, sizeof(float) * count * rr::IN, cudaMemcpyHostToDevice, m->s));
    RR_CUDA(cudaMemcpyAsync(m->y.p, y, sizeof(float) * count, cudaMemcpyHostToDevice, m->s));
    std::vector<int64_t> perm(static_cast<size_t>(count));
    std::iota(perm.begin(), perm.end(), 0);
    uint64_t st = shuffle_seed;
    std::vector<float> losses(static_cast<size_t>(count / bsz + 1));
    for (int ep = 0; ep < epochs; ++ep) {
      for (int64_t i = count - 1; i > 0; --i) {  // Fisher-Yates
        const int64_t j = static_cast<int64_t>(rr::splitmix(st) % static_cast<uint64_t>(i + 1));
        std::swap(perm[static_cast<size_t>(i)], perm[static_cast<size_t>(j)]);
      }
      RR_CUDA(cudaMemcpyAsync(m->idx.p, perm.data(), sizeof(int64_t) * count, cudaMemcpyHostToDevice, m->s));
      double ep_loss = 0.0;
      for (int64_t b0 = 0; b0 < count; b0 += bsz) {
        const int64_t cnt = std::min(bsz, count - b0);
        m->fwd_bwd(m->X.p, m->y.p, m->idx.p + b0, cnt);
        ++m->adam_t;
        const float c1 = 1.0f - std::pow(0.9f, static_cast<float>(m->adam_t));
        const float c2 = 1.0f - std::pow(0.999f, static_cast<float>(m->adam_t));
        rr::adam_f32_kernel<<<(rr::NPARAM + 255) / 256, 256, 0, m->s>>>(m->params.p, m->grad.p, m->m.p, m->v.p,
                                                                         rr::NPARAM, learning_rate, c1, c2);
        RR_LAUNCH_CHECK();
        float l;
        RR_CUDA(cudaMemcpyAsync(&l, m->scal.p, sizeof(float), cudaMemcpyDeviceToHost, m->s));
        RR_CUDA(cudaStreamSynchronize(m->s));
        ep_loss += l;
      }
      if (loss_per_epoch) loss_per_epoch[ep] = static_cast<float>(ep_loss / static_cast<double>(count));
    }
    RR_CUDA(cudaStreamSynchronize(m->s));
  });
}

int rr_mlp_predict(rr_mlp_handle h, const float* X, int64_t count, int32_t bf16, float* y) {
  return mlp_guard([&] {
    auto* m = checked_mlp(h);
    RR_REQUIRE(X && y && count >= 0, RR_ERR_ARG, "rr_mlp_predict: bad arguments");
    if (count == 0) return;
    rr::DevBuf<float> xd(static_cast<size_t>(count * rr::IN)), yd(static_cast<size_t>(count));
    RR_CUDA(cudaMemcpyAsync(xd.p, X, sizeof(float) * count * rr::IN, cudaMemcpyHostToDevice, m->s));
    const int blocks = static_cast<int>((count + rr::TPB - 1) / rr::TPB);
    if (bf16)
      rr::mlp_forward_kernel<false, true><<<blocks, rr::TPB, 0, m->s>>>(m->params.p, m->norm.p, xd.p, nullptr, count,
                                                                        nullptr, nullptr, nullptr, nullptr, yd.p);
    else
      rr::mlp_forward_kernel<false, false><<<blocks, rr::TPB, 0, m->s>>>(m->params.p, m->norm.p, xd.p, nullptr, count,
                                                                         nullptr, nullptr, nullptr, nullptr, yd.p);
    RR_LAUNCH_CHECK();
    std::vector<float> out(static_cast<size_t>(count));
    RR_CUDA(cudaMemcpyAsync(out.data(), yd.p, sizeof(float) * count, cudaMemcpyDeviceToHost, m->s));
    RR_CUDA(cudaStreamSynchronize(m->s));
    const float mu = m->host_norm[2 * rr::IN], sd = m->host_norm[2 * rr::IN + 1];
    for (int64_t i = 0; i < count; ++i) y[i] = out[static_cast<size_t>(i)] * sd + mu;  // back to label units
  });
}

int rr_mlp_loss_and_grad(rr_mlp_handle h, const float* X, const float* y, int64_t count, float* loss, float* grad) {
  return mlp_guard([&] {
    auto* m = checked_mlp(h);
    RR_REQUIRE(X && y && count > 0 && loss && grad, RR_ERR_ARG, "rr_mlp_loss_and_grad: bad arguments");
    m->ensure_scratch(count, count);
    RR_CUDA(cudaMemcpyAsync(m->X.p, X, sizeof(float) * count * rr::IN, cudaMemcpyHostToDevice, m->s));
    RR_CUDA(cudaMemcpyAsync(m->y.p, y, sizeof(float) * count, cudaMemcpyHostToDevice, m->s));
    m->fwd_bwd(m->X.p, m->y.p, nullptr, count);
    float l;
    RR_CUDA(cudaMemcpyAsync(&l, m->scal.p, sizeof(float), cudaMemcpyDeviceToHost, m->s));
    RR_CUDA(cudaMemcpyAsync(grad, m->grad.p, sizeof(float) * rr::NPARAM, cudaMemcpyDeviceToHost, m->s));
    RR_CUDA(cudaStreamSynchronize(m->s));
    *loss = l / static_cast<float>(count);
  });
}

int rr_mlp_get_params(rr_mlp_handle h, float* params) {
  return mlp_guard([&] {
    auto* m = checked_mlp(h);
    RR_REQUIRE(params, RR_ERR_ARG, "rr_mlp_get_params: null output");
    RR_CUDA(cudaMemcpy(params, m->params.p, sizeof(float) * rr::NPARAM, cudaMemcpyDeviceToHost));
    std::memcpy(params + rr::NPARAM, m->host_norm.data(), sizeof(float) * rr::NNORM);
  });
}

int rr_mlp_set_params(rr_mlp_handle h, const float* params) {
  return mlp_guard([&] {
    auto* m = checked_mlp(h);
    RR_REQUIRE(params, RR_ERR_ARG, "rr_mlp_set_params: null input");
    RR_CUDA(cudaMemcpy(m->params.p, params, sizeof(float) * rr::NPARAM, cudaMemcpyHostToDevice));
    m->host_norm.assign(params + rr::NPARAM, params + rr::NPARAM + rr::NNORM);
    RR_CUDA(cudaMemcpy(m->norm.p, m->host_norm.data(), sizeof(float) * rr::NNORM, cudaMemcpyHostToDevice));
    m->has_norm = true;
  });
}

}  // extern "C"
