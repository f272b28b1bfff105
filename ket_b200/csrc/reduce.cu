// reduce.cu -- FP64 reductions over the state: norm, inner product, batched
// Pauli-string expectations, and the fixed-tree Born-rule sampler.
//
// Replaces
//   ket::expval(State, pauli)        src/observable.cpp:18-83
//   ket::expval(State, PauliSum)     src/observable.cpp:85-91
//   ket::measure(State, rng)         src/measurement.cpp:12-21
// The reference runs one serial pass per Pauli term and one O(2^n) scan per
// shot.  Here every term of a sum shares one launch (each term re-reads the
// state through XOR-permuted but coalesced loads), and sampling builds one
// FP64 CDF tree per state and answers all shots with a short descent each.
// All sums are deterministic: fixed per-thread order, fixed warp/block trees,
// block partials reduced in index order by a second kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <type_traits>
#include <cstring>
#include <vector>

#include "internal.h"

namespace kb {
namespace {

constexpr int kRThreads = 256;

template <typename T>
struct AmpT;
template <>
struct AmpT<float2> {
  static __device__ __forceinline__ double re(float2 v) { return (double)v.x; }
  static __device__ __forceinline__ double im(float2 v) { return (double)v.y; }
};
template <>
struct AmpT<double2> {
  static __device__ __forceinline__ double re(double2 v) { return v.x; }
  static __device__ __forceinline__ double im(double2 v) { return v.y; }
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block sum in a fixed tree; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double r = 0;
  if (warp == 0) {
    r = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;
}

template <typename T>
__global__ void norm_partial(const T* __restrict__ s, uint64_t dim, double* __restrict__ part) {
  __shared__ double sh[32];
  double acc = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < dim;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const T v = s[i];
    const double x = AmpT<T>::re(v), y = AmpT<T>::im(v);
    acc += x * x + y * y;
  }
  const double r = block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

template <typename T>
__global__ void inner_partial(const T* __restrict__ a, const T* __restrict__ b, uint64_t dim,
                              double* __restrict__ part) {
  __shared__ double sh[32];
  double re = 0, im = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < dim;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const T u = a[i], v = b[i];
    const double ur = AmpT<T>::re(u), ui = AmpT<T>::im(u);
    const double vr = AmpT<T>::re(v), vi = AmpT<T>::im(v);
    re += ur * vr + ui * vi;  // conj(u) * v
    im += ur * vi - ui * vr;
  }
  const double r0 = block_sum(re, sh);
  const double r1 = block_sum(im, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = r0;
    part[2 * blockIdx.x + 1] = r1;
  }
}

// Mixed-precision comparison: max |a-b| and the sums <a|b>, <a|a>, <b|b>.
template <typename TA, typename TB>
__global__ void compare_partial(const TA* __restrict__ a, const TB* __restrict__ b, uint64_t dim,
                                double* __restrict__ part /* 5 per block */) {
  __shared__ double sh[32];
  double re = 0, im = 0, na = 0, nb = 0, mx = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < dim;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const TA u = a[i];
    const TB v = b[i];
    const double ur = AmpT<TA>::re(u), ui = AmpT<TA>::im(u);
    const double vr = AmpT<TB>::re(v), vi = AmpT<TB>::im(v);
    re += ur * vr + ui * vi;
    im += ur * vi - ui * vr;
    na += ur * ur + ui * ui;
    nb += vr * vr + vi * vi;
    mx = fmax(mx, fmax(fabs(ur - vr), fabs(ui - vi)));
  }
  const double r0 = block_sum(re, sh), r1 = block_sum(im, sh), r2 = block_sum(na, sh), r3 = block_sum(nb, sh);
  // block max
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  if (lane == 0) sh[warp] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, sh[w]);
    part[5 * blockIdx.x + 0] = m;
    part[5 * blockIdx.x + 1] = r0;
    part[5 * blockIdx.x + 2] = r1;
    part[5 * blockIdx.x + 3] = r2;
    part[5 * blockIdx.x + 4] = r3;
  }
}

// Sum `count` partials of `width` interleaved values each, in index order.
__global__ void finish_partials(const double* __restrict__ part, int count, int width,
                                double* __restrict__ out) {
  __shared__ double sh[32];
  for (int w = 0; w < width; ++w) {
    double acc = 0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) acc += part[(size_t)i * width + w];
    const double r = block_sum(acc, sh);
    if (threadIdx.x == 0) out[w] = r;
  }
}

// Batched Pauli terms.  Term t: flip f, sign mask s, phase i^q.  Contribution
// of x: Re(i^q (-1)^popcount(x&s) psi[x] conj(psi[x^f])).  blockIdx.y picks
// a batch of up to kTermBatch terms.
constexpr int kTermBatch = 8;
constexpr int kXPerThread = 4;

struct TermArgs {
  uint64_t flip[kTermBatch];
  uint64_t sign[kTermBatch];
  int q[kTermBatch];
  int count;
};

template <typename T>
__global__ void __launch_bounds__(kRThreads)
    expval_partial(const T* __restrict__ s, uint64_t dim, const uint64_t* __restrict__ flips,
                   const uint64_t* __restrict__ signs, const int* __restrict__ qs, int n_terms,
                   double* __restrict__ part /* [term][block] */) {
  __shared__ double sh[32];
  const int t0 = blockIdx.y * kTermBatch;
  const uint64_t chunk = (uint64_t)kRThreads * kXPerThread;
  const uint64_t nblk = (dim + chunk - 1) / chunk;
  double acc[kTermBatch];
#pragma unroll
  for (int t = 0; t < kTermBatch; ++t) acc[t] = 0;
  for (uint64_t blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
    T a[kXPerThread];
    uint64_t xs[kXPerThread];
#pragma unroll
    for (int e = 0; e < kXPerThread; ++e) {
      xs[e] = blk * chunk + threadIdx.x + (uint64_t)e * kRThreads;
      if (xs[e] < dim) a[e] = s[xs[e]];
    }
#pragma unroll
    for (int t = 0; t < kTermBatch; ++t) {
      if (t0 + t >= n_terms) break;
      const uint64_t f = flips[t0 + t], sg = signs[t0 + t];
      const int q = qs[t0 + t];
#pragma unroll
      for (int e = 0; e < kXPerThread; ++e) {
        if (xs[e] >= dim) continue;
        const T b = s[xs[e] ^ f];
        const double ar = AmpT<T>::re(a[e]), ai = AmpT<T>::im(a[e]);
        const double br = AmpT<T>::re(b), bi = AmpT<T>::im(b);
        const double zr = ar * br + ai * bi;
        const double zi = ai * br - ar * bi;
        double v = (q == 0) ? zr : (q == 1) ? -zi : (q == 2) ? -zr : zi;
        if (__popcll(xs[e] & sg) & 1) v = -v;
        acc[t] += v;
      }
    }
  }
#pragma unroll
  for (int t = 0; t < kTermBatch; ++t) {
    if (t0 + t >= n_terms) break;
    const double r = block_sum(acc[t], sh);
    if (threadIdx.x == 0) part[(size_t)(t0 + t) * gridDim.x + blockIdx.x] = r;
  }
}

// ---------------------------------------------------------------------------
// Fixed-tree sampler.  p_i = re*re + im*im in FP64 (round-to-nearest on each
// product and the sum, no fused multiply-add).  Level 1 holds sequential sums
// of 32 consecutive p_i; level l+1 holds sequential sums of 32 consecutive
// level-l values; the top level has at most 32 entries.  Carries are then
// folded top-down in place: F_l[j] = F_{l+1}[parent-1] (or 0) + V_l[first
// child] + ... + V_l[j], each addition rounded in order.  A draw descends:
// at each level the first child with u < F, else the last child.
constexpr int kSeg = 32;
constexpr int kSegThreads = 128;  // 4 warps: 4 x 32 x 33 doubles of staging

__device__ __forceinline__ double prob(float2 v) {
  const double x = (double)v.x, y = (double)v.y;
  return __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
}
__device__ __forceinline__ double prob(double2 v) {
  return __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y));
}

// One warp produces 32 segment sums; each lane folds one segment from shared
// memory after a coalesced, transposing load.
template <typename T, bool LEAF>
__global__ void __launch_bounds__(kSegThreads)
    seg_sums(const T* __restrict__ src, uint64_t n_src, double* __restrict__ dst, uint64_t n_dst) {
  __shared__ double sh[kSegThreads / 32][32][33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t warps_total = (uint64_t)gridDim.x * (kSegThreads / 32);
  for (uint64_t wseg = (uint64_t)blockIdx.x * (kSegThreads / 32) + warp; wseg * 32 < n_dst;
       wseg += warps_total) {
    const uint64_t base = wseg * 32 * kSeg;
#pragma unroll 4
    for (int r = 0; r < 32; ++r) {
      const uint64_t i = base + (uint64_t)r * 32 + lane;
      double v = 0;
      if (i < n_src) {
        if constexpr (LEAF) v = prob(src[i]);
        else v = reinterpret_cast<const double*>(src)[i];
      }
      sh[warp][r][lane] = v;
    }
    __syncwarp();
    const uint64_t j = wseg * 32 + lane;
    if (j < n_dst) {
      double acc = 0;
      const uint64_t lo = j * kSeg;
      for (int c = 0; c < kSeg; ++c)
        if (lo + c < n_src) acc = __dadd_rn(acc, sh[warp][lane][c]);
      dst[j] = acc;
    }
    __syncwarp();
  }
}

__global__ void top_fold(double* v, uint64_t n) {
  double c = 0;
  for (uint64_t j = 0; j < n; ++j) {
    c = __dadd_rn(c, v[j]);
    v[j] = c;
  }
}

// Fold carries into level l (in place) from the inclusive carries of level l+1.
__global__ void __launch_bounds__(kSegThreads)
    down_fold(double* __restrict__ v, uint64_t n, const double* __restrict__ parent, uint64_t n_parent) {
  __shared__ double sh[kSegThreads / 32][32][33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t warps_total = (uint64_t)gridDim.x * (kSegThreads / 32);
  for (uint64_t wp = (uint64_t)blockIdx.x * (kSegThreads / 32) + warp; wp * 32 < n_parent;
       wp += warps_total) {
    const uint64_t base = wp * 32 * kSeg;
    for (int r = 0; r < 32; ++r) {
      const uint64_t i = base + (uint64_t)r * 32 + lane;
      sh[warp][r][lane] = i < n ? v[i] : 0.0;
    }
    __syncwarp();
    const uint64_t jp = wp * 32 + lane;
    if (jp < n_parent) {
      double c = jp == 0 ? 0.0 : parent[jp - 1];
      const uint64_t lo = jp * kSeg;
      for (int k = 0; k < kSeg; ++k)
        if (lo + k < n) {
          c = __dadd_rn(c, sh[warp][lane][k]);
          sh[warp][lane][k] = c;
        }
    }
    __syncwarp();
    for (int r = 0; r < 32; ++r) {
      const uint64_t i = base + (uint64_t)r * 32 + lane;
      if (i < n) v[i] = sh[warp][r][lane];
    }
    __syncwarp();
  }
}

struct Levels {
  int L;
  uint64_t size[24];
  uint64_t off[24];  // offset (in doubles) of level l >= 1 in the buffer
};

template <typename T>
__global__ void sample_kernel(const T* __restrict__ s, const double* __restrict__ buf, Levels lv,
                              const double* __restrict__ u, uint64_t count, uint64_t* __restrict__ out) {
  const uint64_t d = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= count) return;
  const double x = u[d];
  double carry = 0;
  uint64_t lo = 0, hi = lv.size[lv.L];
  for (int l = lv.L; l >= 1; --l) {
    const double* F = buf + lv.off[l];
    // first j in [lo, hi) with x < F[j] (F non-decreasing within the range)
    uint64_t a = lo, b = hi;
    while (a < b) {
      const uint64_t m = (a + b) >> 1;
      if (x < F[m]) b = m;
      else a = m + 1;
    }
    const uint64_t pick = a < hi ? a : hi - 1;
    if (pick != lo) carry = F[pick - 1];
    lo = pick * kSeg;
    hi = lo + kSeg < lv.size[l - 1] ? lo + kSeg : lv.size[l - 1];
  }
  uint64_t pick = hi - 1;
  double c = carry;
  for (uint64_t i = lo; i < hi; ++i) {
    c = __dadd_rn(c, prob(s[i]));
    if (x < c) {
      pick = i;
      break;
    }
  }
  out[d] = pick;
}

int grid_for(uint64_t work, int per_block) {
  uint64_t g = (work + per_block - 1) / per_block;
  if (g > 148ull * 16) g = 148ull * 16;
  if (g < 1) g = 1;
  return (int)g;
}

// Scratch owned by the call (stream-ordered).
struct Scratch {
  void* p = nullptr;
  cudaStream_t st;
  Scratch(size_t bytes, cudaStream_t s) : st(s) { KB_CUDA(cudaMallocAsync(&p, bytes ? bytes : 8, s)); }
  ~Scratch() {
    if (p) cudaFreeAsync(p, st);
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

template <typename T>
__global__ void rescale_kernel(T* __restrict__ s, uint64_t dim, const double* __restrict__ target,
                               const double* __restrict__ current) {
  const double c = current[0];
  const double f = c > 0.0 ? sqrt(target[0] / c) : 1.0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if constexpr (std::is_same_v<T, float2>) {
    // complex64: two amplitudes per 16-byte access, four accesses in flight;
    // x * f = fma(x, f - 1, x) in FP32 rounds once, like the FP64 product
    // rounded to FP32 (f - 1 is small, so its own FP32 rounding is far below
    // an ulp of x)
    const float d = (float)(f - 1.0);
    float4* s4 = reinterpret_cast<float4*>(s);
    const uint64_t n4 = dim / 2;
    auto scale = [d](float4 v) {
      return make_float4(fmaf(v.x, d, v.x), fmaf(v.y, d, v.y), fmaf(v.z, d, v.z), fmaf(v.w, d, v.w));
    };
    for (; i + 3 * stride < n4; i += 4 * stride) {
      float4 v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) v[u] = s4[i + u * stride];
#pragma unroll
      for (int u = 0; u < 4; ++u) s4[i + u * stride] = scale(v[u]);
    }
    for (; i < n4; i += stride) s4[i] = scale(s4[i]);
    if ((dim & 1) && blockIdx.x == 0 && threadIdx.x == 0) {  // a 1-amplitude state
      s[dim - 1].x = fmaf(s[dim - 1].x, d, s[dim - 1].x);
      s[dim - 1].y = fmaf(s[dim - 1].y, d, s[dim - 1].y);
    }
  } else {
    for (; i < dim; i += stride) {
      T v = s[i];
      v.x = v.x * f;
      v.y = v.y * f;
      s[i] = v;
    }
  }
}

}  // namespace

void norm_to_device(const State& st, double* partials, double* out) {
  if (st.precision == KETGPU_C64)
    norm_partial<float2><<<kNormBlocks, kRThreads, 0, st.stream>>>(static_cast<const float2*>(st.amps), st.dim(),
                                                                   partials);
  else
    norm_partial<double2><<<kNormBlocks, kRThreads, 0, st.stream>>>(static_cast<const double2*>(st.amps), st.dim(),
                                                                    partials);
  finish_partials<<<1, kRThreads, 0, st.stream>>>(partials, kNormBlocks, 1, out);
  count_launch(2);
  KB_CUDA(cudaGetLastError());
}

void norm_from_partials(const State& st, const double* partials, double* out) {
  finish_partials<<<1, kRThreads, 0, st.stream>>>(partials, kNormBlocks, 1, out);
  count_launch();
  KB_CUDA(cudaGetLastError());
}

void rescale_state(const State& st, const double* target, const double* current) {
  if (st.precision == KETGPU_C64)
    rescale_kernel<float2><<<kNormBlocks, kRThreads, 0, st.stream>>>(static_cast<float2*>(st.amps), st.dim(),
                                                                     target, current);
  else
    rescale_kernel<double2><<<kNormBlocks, kRThreads, 0, st.stream>>>(static_cast<double2*>(st.amps), st.dim(),
                                                                      target, current);
  count_launch();
  KB_CUDA(cudaGetLastError());
}

double reduce_norm(const State& st) {
  const int blocks = grid_for(st.dim(), kRThreads * 8);
  Scratch part(sizeof(double) * (blocks + 1), st.stream);
  double* d = part.as<double>();
  if (st.precision == KETGPU_C64)
    norm_partial<float2><<<blocks, kRThreads, 0, st.stream>>>(static_cast<const float2*>(st.amps), st.dim(), d);
  else
    norm_partial<double2><<<blocks, kRThreads, 0, st.stream>>>(static_cast<const double2*>(st.amps), st.dim(), d);
  finish_partials<<<1, kRThreads, 0, st.stream>>>(d, blocks, 1, d + blocks);
  count_launch(2);
  KB_CUDA(cudaGetLastError());
  double h = 0;
  KB_CUDA(cudaMemcpyAsync(&h, d + blocks, sizeof(double), cudaMemcpyDeviceToHost, st.stream));
  KB_CUDA(cudaStreamSynchronize(st.stream));
  return h;
}

cplx reduce_inner(const State& a, const State& b) {
  const int blocks = grid_for(a.dim(), kRThreads * 8);
  Scratch part(sizeof(double) * 2 * (blocks + 1), a.stream);
  double* d = part.as<double>();
  if (b.stream != a.stream) KB_CUDA(cudaStreamSynchronize(b.stream));
  if (a.precision == KETGPU_C64)
    inner_partial<float2><<<blocks, kRThreads, 0, a.stream>>>(static_cast<const float2*>(a.amps),
                                                              static_cast<const float2*>(b.amps), a.dim(), d);
  else
    inner_partial<double2><<<blocks, kRThreads, 0, a.stream>>>(static_cast<const double2*>(a.amps),
                                                               static_cast<const double2*>(b.amps), a.dim(), d);
  finish_partials<<<1, kRThreads, 0, a.stream>>>(d, blocks, 2, d + 2 * blocks);
  count_launch(2);
  KB_CUDA(cudaGetLastError());
  double h[2];
  KB_CUDA(cudaMemcpyAsync(h, d + 2 * blocks, sizeof h, cudaMemcpyDeviceToHost, a.stream));
  KB_CUDA(cudaStreamSynchronize(a.stream));
  return {h[0], h[1]};
}

void compare_states(const State& a, const State& b, double out[5]) {
  const int blocks = grid_for(a.dim(), kRThreads * 8);
  Scratch part(sizeof(double) * 5 * blocks, a.stream);
  double* d = part.as<double>();
  KB_CUDA(cudaStreamSynchronize(b.stream));
  const bool a64 = a.precision == KETGPU_C64, b64 = b.precision == KETGPU_C64;
  if (a64 && b64)
    compare_partial<float2, float2><<<blocks, kRThreads, 0, a.stream>>>(
        static_cast<const float2*>(a.amps), static_cast<const float2*>(b.amps), a.dim(), d);
  else if (a64)
    compare_partial<float2, double2><<<blocks, kRThreads, 0, a.stream>>>(
        static_cast<const float2*>(a.amps), static_cast<const double2*>(b.amps), a.dim(), d);
  else if (b64)
    compare_partial<double2, float2><<<blocks, kRThreads, 0, a.stream>>>(
        static_cast<const double2*>(a.amps), static_cast<const float2*>(b.amps), a.dim(), d);
  else
    compare_partial<double2, double2><<<blocks, kRThreads, 0, a.stream>>>(
        static_cast<const double2*>(a.amps), static_cast<const double2*>(b.amps), a.dim(), d);
  count_launch();
  KB_CUDA(cudaGetLastError());
  std::vector<double> h((size_t)5 * blocks);
  KB_CUDA(cudaMemcpyAsync(h.data(), d, h.size() * sizeof(double), cudaMemcpyDeviceToHost, a.stream));
  KB_CUDA(cudaStreamSynchronize(a.stream));
  for (int w = 0; w < 5; ++w) out[w] = 0;
  for (int bl = 0; bl < blocks; ++bl) {
    out[0] = std::max(out[0], h[5 * bl]);
    for (int w = 1; w < 5; ++w) out[w] += h[5 * bl + w];
  }
}

void expval_terms(const State& st, const std::vector<uint64_t>& flip, const std::vector<uint64_t>& sign,
                  const std::vector<int>& phase, double* out) {
  const int T = (int)flip.size();
  if (T == 0) return;
  const int bx = grid_for(st.dim(), kRThreads * kXPerThread);
  const int by = (T + kTermBatch - 1) / kTermBatch;
  const size_t meta = sizeof(uint64_t) * 2 * T + sizeof(int) * T;
  const size_t parts = sizeof(double) * ((size_t)T * bx + T);
  Scratch sc(meta + parts + 64, st.stream);
  char* base = sc.as<char>();
  uint64_t* d_flip = reinterpret_cast<uint64_t*>(base);
  uint64_t* d_sign = d_flip + T;
  int* d_q = reinterpret_cast<int*>(d_sign + T);
  double* d_part = reinterpret_cast<double*>(base + ((meta + 15) / 16) * 16);
  std::vector<char> host(meta);
  std::memcpy(host.data(), flip.data(), sizeof(uint64_t) * T);
  std::memcpy(host.data() + sizeof(uint64_t) * T, sign.data(), sizeof(uint64_t) * T);
  std::memcpy(host.data() + sizeof(uint64_t) * 2 * T, phase.data(), sizeof(int) * T);
  KB_CUDA(cudaMemcpyAsync(base, host.data(), meta, cudaMemcpyHostToDevice, st.stream));
  dim3 grid(bx, by);
  if (st.precision == KETGPU_C64)
    expval_partial<float2><<<grid, kRThreads, 0, st.stream>>>(static_cast<const float2*>(st.amps), st.dim(),
                                                              d_flip, d_sign, d_q, T, d_part);
  else
    expval_partial<double2><<<grid, kRThreads, 0, st.stream>>>(static_cast<const double2*>(st.amps), st.dim(),
                                                               d_flip, d_sign, d_q, T, d_part);
  count_launch();
  double* d_out = d_part + (size_t)T * bx;
  for (int t = 0; t < T; ++t) {
    finish_partials<<<1, kRThreads, 0, st.stream>>>(d_part + (size_t)t * bx, bx, 1, d_out + t);
    count_launch();
  }
  KB_CUDA(cudaGetLastError());
  KB_CUDA(cudaMemcpyAsync(out, d_out, sizeof(double) * T, cudaMemcpyDeviceToHost, st.stream));
  KB_CUDA(cudaStreamSynchronize(st.stream));
}

std::atomic<uint64_t> g_tree_builds{0};

uint64_t sample_tree_builds() { return g_tree_builds.load(); }

void sample_tree(const State& st, const double* u, uint64_t count, uint64_t* out) {
  Levels lv{};
  lv.size[0] = st.dim();
  lv.L = 0;
  uint64_t total = 0;
  while (lv.size[lv.L] > (uint64_t)kSeg) {
    lv.size[lv.L + 1] = (lv.size[lv.L] + kSeg - 1) / kSeg;
    ++lv.L;
    lv.off[lv.L] = total;
    total += lv.size[lv.L];
  }
  // The tree lives with the state (1/31 of a complex128 state's size, 1/15
  // of a complex64 one) and is rebuilt only after the amplitudes changed.
  if (total && !st.tree) {
    KB_CUDA(cudaMalloc(&st.tree, sizeof(double) * total));
    st.tree_doubles = total;
  }
  const size_t ubytes = sizeof(double) * count, obytes = sizeof(uint64_t) * count;
  Scratch sc(ubytes + obytes + 64, st.stream);
  double* buf = st.tree;
  double* d_u = sc.as<double>();
  uint64_t* d_out = reinterpret_cast<uint64_t*>(d_u + count);
  KB_CUDA(cudaMemcpyAsync(d_u, u, ubytes, cudaMemcpyHostToDevice, st.stream));
  const bool build = total && st.tree_version != st.version;
  if (build) g_tree_builds.fetch_add(1);
  for (int l = 1; build && l <= lv.L; ++l) {
    const uint64_t nd = lv.size[l];
    const int blocks = grid_for(nd, kSegThreads);  // one warp -> 32 outputs
    if (l == 1) {
      if (st.precision == KETGPU_C64)
        seg_sums<float2, true><<<blocks, kSegThreads, 0, st.stream>>>(static_cast<const float2*>(st.amps),
                                                                      lv.size[0], buf + lv.off[1], nd);
      else
        seg_sums<double2, true><<<blocks, kSegThreads, 0, st.stream>>>(static_cast<const double2*>(st.amps),
                                                                       lv.size[0], buf + lv.off[1], nd);
    } else {
      seg_sums<double, false><<<blocks, kSegThreads, 0, st.stream>>>(buf + lv.off[l - 1], lv.size[l - 1],
                                                                     buf + lv.off[l], nd);
    }
    count_launch();
  }
  if (build) {
    top_fold<<<1, 1, 0, st.stream>>>(buf + lv.off[lv.L], lv.size[lv.L]);
    count_launch();
    for (int l = lv.L - 1; l >= 1; --l) {
      const int blocks = grid_for(lv.size[l + 1], kSegThreads);
      down_fold<<<blocks, kSegThreads, 0, st.stream>>>(buf + lv.off[l], lv.size[l], buf + lv.off[l + 1],
                                                     lv.size[l + 1]);
      count_launch();
    }
  }
  const int blocks = (int)((count + kRThreads - 1) / kRThreads);
  if (count) {
    if (st.precision == KETGPU_C64)
      sample_kernel<float2><<<blocks, kRThreads, 0, st.stream>>>(static_cast<const float2*>(st.amps), buf, lv,
                                                                 d_u, count, d_out);
    else
      sample_kernel<double2><<<blocks, kRThreads, 0, st.stream>>>(static_cast<const double2*>(st.amps), buf, lv,
                                                                  d_u, count, d_out);
    count_launch();
  }
  KB_CUDA(cudaGetLastError());
  if (build) st.tree_version = st.version;
  KB_CUDA(cudaMemcpyAsync(out, d_out, obytes, cudaMemcpyDeviceToHost, st.stream));
  KB_CUDA(cudaStreamSynchronize(st.stream));
}

}  // namespace kb
