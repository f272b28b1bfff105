// mlp.cu -- the learned fusion cost model: a 48 -> 128 -> 128 -> 1 ReLU MLP
// with BF16 weights and FP32 accumulation, trained on the GPU with
// hand-written forward, backward and Adam kernels.
//
// No ket counterpart (ket's Fuser, src/simulator.cpp:400-477, uses a fixed
// rule).  The model regresses log(pass time in microseconds) from the 48
// pass features of planner.cpp; the learned planner scores candidate
// partitions with it (one batched inference per circuit segment).
//
// Parameter layout (one contiguous vector, FP32 masters + BF16 copies):
//   W1 [128][48] | b1 [128] | W2 [128][128] | b2 [128] | w3 [128] | b3 [1]
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <random>
#include <vector>

#include "internal.h"

#define KB_API extern "C" __attribute__((visibility("default")))

namespace kb {
namespace {

constexpr int IN = KETGPU_MLP_IN, HID = KETGPU_MLP_HIDDEN;
constexpr size_t OFF_W1 = 0, OFF_B1 = OFF_W1 + HID * IN, OFF_W2 = OFF_B1 + HID, OFF_B2 = OFF_W2 + HID * HID,
                 OFF_W3 = OFF_B2 + HID, OFF_B3 = OFF_W3 + HID, NPARAM = OFF_B3 + 1;
constexpr int TILE_S = 16;  // samples per CTA

struct Mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  float* master = nullptr;
  __nv_bfloat16* w = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  float* grad = nullptr;
  float* loss = nullptr;
  int step = 0;
  // scratch grown on demand
  float* xbuf = nullptr;
  float* ybuf = nullptr;
  float* act = nullptr;
  float* out = nullptr;
  int* idx = nullptr;
  size_t cap = 0;
};

__device__ __forceinline__ float bf(const __nv_bfloat16* w, size_t i) { return __bfloat162float(w[i]); }

// out[s] = w3 . relu(W2 relu(W1 x_s + b1) + b2) + b3 for the tile's samples;
// act (optional) keeps z1 | z2 per sample for the backward pass.
__global__ void __launch_bounds__(HID)
    mlp_fwd(const __nv_bfloat16* __restrict__ w, const float* __restrict__ x, const int* __restrict__ idx,
            int batch, float* __restrict__ out, float* __restrict__ act) {
  __shared__ float xs[TILE_S][IN];
  __shared__ float h1[TILE_S][HID];
  __shared__ float red[TILE_S][HID / 32];
  const int i = threadIdx.x, s0 = blockIdx.x * TILE_S;
  for (int e = i; e < TILE_S * IN; e += HID) {
    const int s = e / IN, k = e % IN;
    const int row = s0 + s < batch ? (idx ? idx[s0 + s] : s0 + s) : -1;
    xs[s][k] = row >= 0 ? x[(size_t)row * IN + k] : 0.f;
  }
  __syncthreads();
  float w1r[IN];
#pragma unroll
  for (int k = 0; k < IN; ++k) w1r[k] = bf(w, OFF_W1 + (size_t)i * IN + k);
  const float b1 = bf(w, OFF_B1 + i), b2 = bf(w, OFF_B2 + i), w3 = bf(w, OFF_W3 + i);
  for (int s = 0; s < TILE_S; ++s) {
    float z = b1;
#pragma unroll
    for (int k = 0; k < IN; ++k) z = fmaf(w1r[k], xs[s][k], z);
    h1[s][i] = fmaxf(z, 0.f);
    if (act && s0 + s < batch) act[(size_t)(s0 + s) * 2 * HID + i] = z;
  }
  __syncthreads();
  const __nv_bfloat162* w2 = reinterpret_cast<const __nv_bfloat162*>(w + OFF_W2 + (size_t)i * HID);
  for (int s = 0; s < TILE_S; ++s) {
    float z = b2;
#pragma unroll 8
    for (int k = 0; k < HID / 2; ++k) {
      const float2 wv = __bfloat1622float2(w2[k]);
      z = fmaf(wv.x, h1[s][2 * k], z);
      z = fmaf(wv.y, h1[s][2 * k + 1], z);
    }
    if (act && s0 + s < batch) act[(size_t)(s0 + s) * 2 * HID + HID + i] = z;
    float c = w3 * fmaxf(z, 0.f);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((i & 31) == 0) red[s][i >> 5] = c;
  }
  __syncthreads();
  if (i < TILE_S && s0 + i < batch) {
    float t = bf(w, OFF_B3);
    for (int k = 0; k < HID / 32; ++k) t += red[i][k];
    out[s0 + i] = t;
  }
}

// Gradients of L = mean_s (out_s - y_s)^2, accumulated into grad (FP32).
__global__ void __launch_bounds__(HID)
    mlp_bwd(const __nv_bfloat16* __restrict__ w, const float* __restrict__ x, const float* __restrict__ y,
            const int* __restrict__ idx, const float* __restrict__ act, const float* __restrict__ out, int batch,
            float* __restrict__ grad, float* __restrict__ loss) {
  __shared__ float xs[TILE_S][IN];
  __shared__ float h1[TILE_S][HID];
  __shared__ float d2[TILE_S][HID];
  __shared__ float d1[TILE_S][HID];
  __shared__ float dout[TILE_S];
  const int i = threadIdx.x, s0 = blockIdx.x * TILE_S;
  const int ns = min(TILE_S, batch - s0);
  for (int e = i; e < TILE_S * IN; e += HID) {
    const int s = e / IN, k = e % IN;
    const int row = s < ns ? (idx ? idx[s0 + s] : s0 + s) : -1;
    xs[s][k] = row >= 0 ? x[(size_t)row * IN + k] : 0.f;
  }
  if (i < TILE_S) {
    float d = 0.f;
    if (i < ns) {
      const int row = idx ? idx[s0 + i] : s0 + i;
      const float e = out[s0 + i] - y[row];
      d = 2.f * e / (float)batch;
      atomicAdd(loss, e * e / (float)batch);
    }
    dout[i] = d;
  }
  for (int s = 0; s < TILE_S; ++s) h1[s][i] = s < ns ? fmaxf(act[(size_t)(s0 + s) * 2 * HID + i], 0.f) : 0.f;
  __syncthreads();
  const float w3 = bf(w, OFF_W3 + i);
  float gw3 = 0.f, gb2 = 0.f;
  for (int s = 0; s < TILE_S; ++s) {
    const float z2 = s < ns ? act[(size_t)(s0 + s) * 2 * HID + HID + i] : 0.f;
    gw3 += dout[s] * fmaxf(z2, 0.f);
    const float d = (z2 > 0.f) ? dout[s] * w3 : 0.f;
    d2[s][i] = d;
    gb2 += d;
  }
  atomicAdd(&grad[OFF_W3 + i], gw3);
  atomicAdd(&grad[OFF_B2 + i], gb2);
  if (i == 0) {
    float gb3 = 0.f;
    for (int s = 0; s < TILE_S; ++s) gb3 += dout[s];
    atomicAdd(&grad[OFF_B3], gb3);
  }
  __syncthreads();
  // gW2[i][k] = sum_s d2[s][i] h1[s][k]
  for (int k = 0; k < HID; ++k) {
    float a = 0.f;
#pragma unroll
    for (int s = 0; s < TILE_S; ++s) a = fmaf(d2[s][i], h1[s][k], a);
    atomicAdd(&grad[OFF_W2 + (size_t)i * HID + k], a);
  }
  // d1[s][k=i] = sum_j d2[s][j] W2[j][i], masked by z1 > 0
  for (int s = 0; s < TILE_S; ++s) {
    float a = 0.f;
    for (int j = 0; j < HID; ++j) a = fmaf(d2[s][j], bf(w, OFF_W2 + (size_t)j * HID + i), a);
    const float z1 = s < ns ? act[(size_t)(s0 + s) * 2 * HID + i] : 0.f;
    d1[s][i] = z1 > 0.f ? a : 0.f;
  }
  __syncthreads();
  float gb1 = 0.f;
  for (int s = 0; s < TILE_S; ++s) gb1 += d1[s][i];
  atomicAdd(&grad[OFF_B1 + i], gb1);
  for (int k = 0; k < IN; ++k) {
    float a = 0.f;
#pragma unroll
    for (int s = 0; s < TILE_S; ++s) a = fmaf(d1[s][i], xs[s][k], a);
    atomicAdd(&grad[OFF_W1 + (size_t)i * IN + k], a);
  }
}

// Adam on the FP32 masters, refreshing the BF16 copies; zeroes the gradient.
__global__ void mlp_adam(float* __restrict__ master, __nv_bfloat16* __restrict__ w, float* __restrict__ m,
                         float* __restrict__ v, float* __restrict__ grad, size_t count, float lr, float c1,
                         float c2) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    const float g = grad[i];
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float p = master[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    master[i] = p;
    w[i] = __float2bfloat16_rn(p);
    grad[i] = 0.f;
  }
}

__global__ void mlp_sync_bf16(const float* __restrict__ master, __nv_bfloat16* __restrict__ w, size_t count) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    w[i] = __float2bfloat16_rn(master[i]);
}

void ensure(Mlp& M, size_t batch, size_t samples) {
  const size_t need = std::max(batch, samples);
  if (need <= M.cap) return;
  cudaFree(M.xbuf);
  cudaFree(M.ybuf);
  cudaFree(M.act);
  cudaFree(M.out);
  cudaFree(M.idx);
  M.xbuf = M.ybuf = M.act = M.out = nullptr;
  M.idx = nullptr;
  KB_CUDA(cudaMalloc(&M.xbuf, need * IN * sizeof(float)));
  KB_CUDA(cudaMalloc(&M.ybuf, need * sizeof(float)));
  KB_CUDA(cudaMalloc(&M.act, need * 2 * HID * sizeof(float)));
  KB_CUDA(cudaMalloc(&M.out, need * sizeof(float)));
  KB_CUDA(cudaMalloc(&M.idx, need * sizeof(int)));
  M.cap = need;
}

void forward(Mlp& M, const float* d_x, const int* d_idx, size_t batch, float* d_out, float* d_act) {
  const unsigned grid = (unsigned)((batch + TILE_S - 1) / TILE_S);
  if (grid) mlp_fwd<<<grid, HID, 0, M.stream>>>(M.w, d_x, d_idx, (int)batch, d_out, d_act);
  count_launch();
  KB_CUDA(cudaGetLastError());
}

void backward(Mlp& M, const float* d_x, const float* d_y, const int* d_idx, size_t batch) {
  const unsigned grid = (unsigned)((batch + TILE_S - 1) / TILE_S);
  if (grid)
    mlp_bwd<<<grid, HID, 0, M.stream>>>(M.w, d_x, d_y, d_idx, M.act, M.out, (int)batch, M.grad, M.loss);
  count_launch();
  KB_CUDA(cudaGetLastError());
}

std::mutex g_model_mu;
Mlp* g_model = nullptr;

}  // namespace

bool learned_model_attached() {
  std::lock_guard<std::mutex> lk(g_model_mu);
  return g_model != nullptr;
}

void learned_predict(const std::vector<float>& rows, std::vector<float>& us) {
  std::lock_guard<std::mutex> lk(g_model_mu);
  if (!g_model) fail(KETGPU_ERR_LOGIC, "no cost model attached");
  Mlp& M = *g_model;
  const size_t batch = rows.size() / kFeatures;
  us.assign(batch, 0.f);
  if (!batch) return;
  DeviceGuard dg(M.device);
  ensure(M, batch, batch);
  KB_CUDA(cudaMemcpyAsync(M.xbuf, rows.data(), rows.size() * sizeof(float), cudaMemcpyHostToDevice, M.stream));
  forward(M, M.xbuf, nullptr, batch, M.out, nullptr);
  KB_CUDA(cudaMemcpyAsync(us.data(), M.out, batch * sizeof(float), cudaMemcpyDeviceToHost, M.stream));
  KB_CUDA(cudaStreamSynchronize(M.stream));
  for (float& u : us) u = std::exp(std::min(u, 30.f));  // the model predicts log(us)
}

}  // namespace kb

using namespace kb;

namespace {
template <class F>
int mlp_guard(F&& f) {
  try {
    f();
    return KETGPU_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return KETGPU_ERR_LOGIC;
  }
}
Mlp* as_mlp(ketgpu_mlp* m) { return reinterpret_cast<Mlp*>(m); }
const Mlp* as_mlp(const ketgpu_mlp* m) { return reinterpret_cast<const Mlp*>(m); }
}  // namespace

KB_API int ketgpu_mlp_create(uint64_t seed, ketgpu_mlp** out) {
  return mlp_guard([&] {
    if (!out) fail(KETGPU_ERR_INVALID, "out is null");
    auto M = std::make_unique<Mlp>();
    KB_CUDA(cudaGetDevice(&M->device));
    KB_CUDA(cudaStreamCreateWithFlags(&M->stream, cudaStreamNonBlocking));
    KB_CUDA(cudaMalloc(&M->master, NPARAM * sizeof(float)));
    KB_CUDA(cudaMalloc(&M->w, NPARAM * sizeof(__nv_bfloat16)));
    KB_CUDA(cudaMalloc(&M->m, NPARAM * sizeof(float)));
    KB_CUDA(cudaMalloc(&M->v, NPARAM * sizeof(float)));
    KB_CUDA(cudaMalloc(&M->grad, NPARAM * sizeof(float)));
    KB_CUDA(cudaMalloc(&M->loss, sizeof(float)));
    // He-uniform initial weights, zero biases
    std::vector<float> h(NPARAM, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](size_t off, size_t cnt, int fan_in) {
      const float lim = std::sqrt(6.f / (float)fan_in);
      std::uniform_real_distribution<float> d(-lim, lim);
      for (size_t i = 0; i < cnt; ++i) h[off + i] = d(rng);
    };
    fill(OFF_W1, HID * IN, IN);
    fill(OFF_W2, HID * HID, HID);
    fill(OFF_W3, HID, HID);
    // on the model's own (non-blocking) stream, ahead of the kernels that
    // read these buffers
    KB_CUDA(cudaMemcpyAsync(M->master, h.data(), NPARAM * sizeof(float), cudaMemcpyHostToDevice, M->stream));
    KB_CUDA(cudaMemsetAsync(M->m, 0, NPARAM * sizeof(float), M->stream));
    KB_CUDA(cudaMemsetAsync(M->v, 0, NPARAM * sizeof(float), M->stream));
    KB_CUDA(cudaMemsetAsync(M->grad, 0, NPARAM * sizeof(float), M->stream));
    mlp_sync_bf16<<<64, 256, 0, M->stream>>>(M->master, M->w, NPARAM);
    count_launch();
    KB_CUDA(cudaStreamSynchronize(M->stream));
    *out = reinterpret_cast<ketgpu_mlp*>(M.release());
  });
}

KB_API int ketgpu_mlp_destroy(ketgpu_mlp* mp) {
  return mlp_guard([&] {
    Mlp* M = as_mlp(mp);
    if (!M) return;
    {
      std::lock_guard<std::mutex> lk(g_model_mu);
      if (g_model == M) g_model = nullptr;
    }
    DeviceGuard dg(M->device);
    cudaStreamSynchronize(M->stream);
    for (void* p : {(void*)M->master, (void*)M->w, (void*)M->m, (void*)M->v, (void*)M->grad, (void*)M->loss,
                    (void*)M->xbuf, (void*)M->ybuf, (void*)M->act, (void*)M->out, (void*)M->idx})
      if (p) cudaFree(p);
    cudaStreamDestroy(M->stream);
    delete M;
  });
}

KB_API int ketgpu_mlp_get_weights(const ketgpu_mlp* mp, float* w1, float* b1, float* w2, float* b2, float* w3,
                                  float* b3) {
  return mlp_guard([&] {
    const Mlp* M = as_mlp(mp);
    if (!M) fail(KETGPU_ERR_INVALID, "model is null");
    DeviceGuard dg(M->device);
    std::vector<__nv_bfloat16> h(NPARAM);
    KB_CUDA(cudaStreamSynchronize(M->stream));  // the model's kernels write M->w on its own stream
    KB_CUDA(cudaMemcpy(h.data(), M->w, NPARAM * sizeof(__nv_bfloat16), cudaMemcpyDeviceToHost));
    auto put = [&](float* dst, size_t off, size_t cnt) {
      if (dst)
        for (size_t i = 0; i < cnt; ++i) dst[i] = __bfloat162float(h[off + i]);
    };
    put(w1, OFF_W1, HID * IN);
    put(b1, OFF_B1, HID);
    put(w2, OFF_W2, HID * HID);
    put(b2, OFF_B2, HID);
    put(w3, OFF_W3, HID);
    put(b3, OFF_B3, 1);
  });
}

KB_API int ketgpu_mlp_set_weights(ketgpu_mlp* mp, const float* w1, const float* b1, const float* w2,
                                  const float* b2, const float* w3, const float* b3) {
  return mlp_guard([&] {
    Mlp* M = as_mlp(mp);
    if (!M || !w1 || !b1 || !w2 || !b2 || !w3 || !b3) fail(KETGPU_ERR_INVALID, "null argument");
    std::vector<float> h(NPARAM);
    std::memcpy(&h[OFF_W1], w1, HID * IN * sizeof(float));
    std::memcpy(&h[OFF_B1], b1, HID * sizeof(float));
    std::memcpy(&h[OFF_W2], w2, HID * HID * sizeof(float));
    std::memcpy(&h[OFF_B2], b2, HID * sizeof(float));
    std::memcpy(&h[OFF_W3], w3, HID * sizeof(float));
    h[OFF_B3] = b3[0];
    DeviceGuard dg(M->device);
    KB_CUDA(cudaMemcpyAsync(M->master, h.data(), NPARAM * sizeof(float), cudaMemcpyHostToDevice, M->stream));
    mlp_sync_bf16<<<64, 256, 0, M->stream>>>(M->master, M->w, NPARAM);
    count_launch();
    KB_CUDA(cudaStreamSynchronize(M->stream));
  });
}

KB_API int ketgpu_mlp_forward(ketgpu_mlp* mp, const float* x, uint64_t batch, float* out) {
  return mlp_guard([&] {
    Mlp* M = as_mlp(mp);
    if (!M || (batch && (!x || !out))) fail(KETGPU_ERR_INVALID, "null argument");
    DeviceGuard dg(M->device);
    ensure(*M, batch, batch);
    KB_CUDA(cudaMemcpyAsync(M->xbuf, x, batch * IN * sizeof(float), cudaMemcpyHostToDevice, M->stream));
    forward(*M, M->xbuf, nullptr, batch, M->out, nullptr);
    KB_CUDA(cudaMemcpyAsync(out, M->out, batch * sizeof(float), cudaMemcpyDeviceToHost, M->stream));
    KB_CUDA(cudaStreamSynchronize(M->stream));
  });
}

KB_API int ketgpu_mlp_gradients(ketgpu_mlp* mp, const float* x, const float* y, uint64_t batch, float* loss,
                                float* gw1, float* gb1, float* gw2, float* gb2, float* gw3, float* gb3) {
  return mlp_guard([&] {
    Mlp* M = as_mlp(mp);
    if (!M || !x || !y || !batch) fail(KETGPU_ERR_INVALID, "null argument");
    DeviceGuard dg(M->device);
    ensure(*M, batch, batch);
    KB_CUDA(cudaMemcpyAsync(M->xbuf, x, batch * IN * sizeof(float), cudaMemcpyHostToDevice, M->stream));
    KB_CUDA(cudaMemcpyAsync(M->ybuf, y, batch * sizeof(float), cudaMemcpyHostToDevice, M->stream));
    KB_CUDA(cudaMemsetAsync(M->grad, 0, NPARAM * sizeof(float), M->stream));
    KB_CUDA(cudaMemsetAsync(M->loss, 0, sizeof(float), M->stream));
    forward(*M, M->xbuf, nullptr, batch, M->out, M->act);
    backward(*M, M->xbuf, M->ybuf, nullptr, batch);
    std::vector<float> g(NPARAM);
    float l = 0.f;
    KB_CUDA(cudaMemcpyAsync(g.data(), M->grad, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, M->stream));
    KB_CUDA(cudaMemcpyAsync(&l, M->loss, sizeof(float), cudaMemcpyDeviceToHost, M->stream));
    KB_CUDA(cudaMemsetAsync(M->grad, 0, NPARAM * sizeof(float), M->stream));
    KB_CUDA(cudaStreamSynchronize(M->stream));
    if (loss) *loss = l;
    auto put = [&](float* dst, size_t off, size_t cnt) {
      if (dst) std::memcpy(dst, &g[off], cnt * sizeof(float));
    };
    put(gw1, OFF_W1, HID * IN);
    put(gb1, OFF_B1, HID);
    put(gw2, OFF_W2, HID * HID);
    put(gb2, OFF_B2, HID);
    put(gw3, OFF_W3, HID);
    put(gb3, OFF_B3, 1);
  });
}

KB_API int ketgpu_mlp_train(ketgpu_mlp* mp, const float* x, const float* y, uint64_t n_samples, uint64_t steps,
                            uint64_t minibatch, float lr, float* final_loss) {
  return mlp_guard([&] {
    Mlp* M = as_mlp(mp);
    if (!M || !x || !y || !n_samples || !minibatch) fail(KETGPU_ERR_INVALID, "null argument");
    DeviceGuard dg(M->device);
    ensure(*M, minibatch, n_samples);
    KB_CUDA(cudaMemcpyAsync(M->xbuf, x, n_samples * IN * sizeof(float), cudaMemcpyHostToDevice, M->stream));
    KB_CUDA(cudaMemcpyAsync(M->ybuf, y, n_samples * sizeof(float), cudaMemcpyHostToDevice, M->stream));
    KB_CUDA(cudaMemsetAsync(M->grad, 0, NPARAM * sizeof(float), M->stream));
    std::mt19937_64 rng(0x5eed + (uint64_t)M->step);
    std::uniform_int_distribution<uint64_t> pick(0, n_samples - 1);
    std::vector<int> idx(minibatch);
    int* pinned = nullptr;
    KB_CUDA(cudaMallocHost(&pinned, minibatch * sizeof(int)));
    float l = 0.f;
    for (uint64_t s = 0; s < steps; ++s) {
      for (auto& i : idx) i = (int)pick(rng);
      KB_CUDA(cudaStreamSynchronize(M->stream));  // the pinned index buffer is reused
      std::memcpy(pinned, idx.data(), minibatch * sizeof(int));
      KB_CUDA(cudaMemcpyAsync(M->idx, pinned, minibatch * sizeof(int), cudaMemcpyHostToDevice, M->stream));
      KB_CUDA(cudaMemsetAsync(M->loss, 0, sizeof(float), M->stream));
      forward(*M, M->xbuf, M->idx, minibatch, M->out, M->act);
      backward(*M, M->xbuf, M->ybuf, M->idx, minibatch);
      ++M->step;
      const float c1 = 1.f - std::pow(0.9f, (float)M->step), c2 = 1.f - std::pow(0.999f, (float)M->step);
      mlp_adam<<<64, 256, 0, M->stream>>>(M->master, M->w, M->m, M->v, M->grad, NPARAM, lr, c1, c2);
      count_launch();
    }
    KB_CUDA(cudaMemcpyAsync(&l, M->loss, sizeof(float), cudaMemcpyDeviceToHost, M->stream));
    KB_CUDA(cudaStreamSynchronize(M->stream));
    cudaFreeHost(pinned);
    if (final_loss) *final_loss = l;
  });
}

KB_API int ketgpu_planner_set_model(ketgpu_mlp* mp) {
  std::lock_guard<std::mutex> lk(g_model_mu);
  g_model = as_mlp(mp);
  return KETGPU_OK;
}

KB_API int ketgpu_block_features(int32_t n, int32_t precision, const ketgpu_op* gates, uint64_t n_gates,
                                 int32_t fused, int32_t tensor, float* out48) {
  return mlp_guard([&] {
    if (!gates || !n_gates || !out48) fail(KETGPU_ERR_INVALID, "null argument");
    validate_ops(n, gates, n_gates);
    std::vector<const ketgpu_op*> gs;
    std::vector<int> qs;
    for (uint64_t i = 0; i < n_gates; ++i) {
      if (!is_unitary(gates[i].type)) continue;
      gs.push_back(&gates[i]);
      for (int j = 0; j < gate_arity(gates[i].type); ++j)
        if (std::find(qs.begin(), qs.end(), gates[i].q[j]) == qs.end()) qs.push_back(gates[i].q[j]);
    }
    if (!fused && gs.size() != 1) fail(KETGPU_ERR_INVALID, "an unfused pass applies exactly one gate");
    pass_features(n, precision, gs, qs, fused != 0, tensor != 0, out48);
  });
}
