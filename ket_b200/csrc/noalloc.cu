// noalloc.cu -- a Pauli-sum expectation that allocates no device memory.
//
// ketgpu_expval_sum (reduce.cu) takes its block partials and term table from
// a stream-ordered allocation made inside the call.  Some callers cannot
// allow that: a service that has reserved nearly all of HBM for resident
// state vectors (an allocation at query time can fail or fragment what is
// left), or a caller that must not let the call allocate and free device
// memory underneath it (cudaMalloc/cudaFree may synchronise the device or
// interfere with the caller's own pool).  ketgpu_expval_sum_noalloc gives
// the same result using only the fixed scratch array below.
//
// The scratch is a file-scope __device__ array: every GPU that loads the
// library holds it (kScratchBytes) until the process exits, and every call
// on a device shares it, keeping the previous call's contents.  Calls whose
// kernels overlap on the same GPU (different streams or threads at once)
// race on it.  Nothing in it needs to start at zero: each call writes every
// partial and every result it reads back.  In host code the array's name is
// only a host-side stand-in, so the device address is looked up once per
// device with cudaGetSymbolAddress, with that device current.
//
// That set-up runs when the first state is created on a device
// (noalloc_prepare, called from create_state), not in the entry point.
// Under CUDA's lazy module loading (the default since CUDA 12.2) this
// module, its scratch array and its kernels are placed on a device only
// when first used, and placing them takes device memory.  Doing it at state
// creation -- which allocates the state anyway -- leaves nothing for the
// entry point itself to allocate.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "internal.h"

#define KB_API extern "C" __attribute__((visibility("default")))

namespace kb {
namespace {

constexpr int kMaxTerms = KETGPU_NOALLOC_MAX_TERMS;
constexpr int kNaBlocks = 296;  // 2 x 148 SMs
constexpr int kNaThreads = 256;
constexpr int kNaPerThread = 4;
// [term][block] partials, then one result per term
constexpr size_t kScratchDoubles = (size_t)kMaxTerms * kNaBlocks + kMaxTerms;
constexpr size_t kScratchBytes = kScratchDoubles * sizeof(double);
static_assert(kScratchBytes == 608256, "the size include/ket_b200.h states");

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Term table passed by value (kernel parameters, 5 KB).
struct TermTable {
  uint64_t flip[kMaxTerms];
  uint64_t sign[kMaxTerms];
  uint8_t q[kMaxTerms];
  int count;
};

template <typename T>
__device__ __forceinline__ double re_of(T v) {
  return (double)v.x;
}
template <typename T>
__device__ __forceinline__ double im_of(T v) {
  return (double)v.y;
}

__device__ __forceinline__ double na_block_sum(double v, double* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double r = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sh[w];
  __syncthreads();
  return r;
}

// Partial sums of Re(i^q (-1)^popcount(x&s) psi[x] conj(psi[x^f])) per term
// and block, written into scratch[t * kNaBlocks + block].
template <typename T>
__global__ void __launch_bounds__(kNaThreads)
    na_partial(const T* __restrict__ s, uint64_t dim, const TermTable tt, double* __restrict__ scratch) {
  __shared__ double sh[32];
  const uint64_t chunk = (uint64_t)kNaThreads * kNaPerThread;
  const uint64_t nchunks = (dim + chunk - 1) / chunk;
  for (int t = 0; t < tt.count; ++t) {
    const uint64_t f = tt.flip[t], sg = tt.sign[t];
    const int q = tt.q[t];
    double acc = 0.0;
    for (uint64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
#pragma unroll
      for (int e = 0; e < kNaPerThread; ++e) {
        const uint64_t x = c * chunk + threadIdx.x + (uint64_t)e * kNaThreads;
        if (x >= dim) continue;
        const T a = s[x], b = s[x ^ f];
        const double ar = re_of(a), ai = im_of(a), br = re_of(b), bi = im_of(b);
        const double zr = ar * br + ai * bi, zi = ai * br - ar * bi;
        double v = (q == 0) ? zr : (q == 1) ? -zi : (q == 2) ? -zr : zi;
        if (__popcll(x & sg) & 1) v = -v;
        acc += v;
      }
    }
    const double r = na_block_sum(acc, sh);
    if (threadIdx.x == 0) scratch[(size_t)t * kNaBlocks + blockIdx.x] = r;
  }
}

// result[t] = sum of the term's block partials, in block order.
__global__ void na_finish(double* __restrict__ scratch, int count) {
  __shared__ double sh[32];
  for (int t = 0; t < count; ++t) {
    double acc = 0.0;
    for (int b = threadIdx.x; b < kNaBlocks; b += blockDim.x) acc += scratch[(size_t)t * kNaBlocks + b];
    const double r = na_block_sum(acc, sh);
    if (threadIdx.x == 0) scratch[(size_t)kMaxTerms * kNaBlocks + t] = r;
  }
}

std::mutex g_na_mu;
double* g_na_ptr[64] = {nullptr};

// Device address of the scratch array on `device` (which must be current).
// The first lookup on a device also loads this module's kernels there
// (cudaFuncGetAttributes), so that a later launch places no code either.
double* scratch_on(int device) {
  if (device < 0 || device >= 64) fail(KETGPU_ERR_INVALID, "expval_sum_noalloc: device index out of range");
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      fail(KETGPU_ERR_CUDA, std::string("expval_sum_noalloc: cudaGetSymbolAddress failed: ") +
                                cudaGetErrorString(e));
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, na_partial<float2>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, na_partial<double2>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, na_finish);
    if (e != cudaSuccess)
      fail(KETGPU_ERR_CUDA, std::string("expval_sum_noalloc: loading its kernels failed: ") + cudaGetErrorString(e));
    g_na_ptr[device] = static_cast<double*>(p);
  }
  return g_na_ptr[device];
}

}  // namespace

void noalloc_prepare(int device) { (void)scratch_on(device); }

}  // namespace kb

using namespace kb;

// Same value as ketgpu_expval_sum, computed in the fixed scratch array (no
// device allocation).  n_terms <= KETGPU_NOALLOC_MAX_TERMS.
KB_API int ketgpu_expval_sum_noalloc(const ketgpu_state* sh, const double* coeffs, const char* const* paulis,
                                     uint64_t n_terms, double* out) {
  try {
    if (!sh || !out) fail(KETGPU_ERR_INVALID, "expval_sum_noalloc: null argument");
    if (n_terms && (!coeffs || !paulis)) fail(KETGPU_ERR_INVALID, "expval_sum_noalloc: null argument");
    if (n_terms > (uint64_t)kMaxTerms)
      fail(KETGPU_ERR_INVALID, "expval_sum_noalloc: " + std::to_string(n_terms) + " terms exceed the fixed scratch (at most " +
                                   std::to_string(kMaxTerms) + " terms; use ketgpu_expval_sum)");
    const State& st = *reinterpret_cast<const State*>(sh);
    TermTable tt;
    std::memset(&tt, 0, sizeof tt);
    tt.count = (int)n_terms;
    for (uint64_t t = 0; t < n_terms; ++t) {
      int q = 0;
      pauli_masks(st.n, paulis[t], tt.flip[t], tt.sign[t], q);
      tt.q[t] = (uint8_t)q;
    }
    *out = 0.0;
    if (n_terms == 0) return KETGPU_OK;
    DeviceGuard g(st.device);
    double* scratch = scratch_on(st.device);
    if (st.precision == KETGPU_C64)
      na_partial<float2><<<kNaBlocks, kNaThreads, 0, st.stream>>>(static_cast<const float2*>(st.amps), st.dim(), tt,
                                                                   scratch);
    else
      na_partial<double2><<<kNaBlocks, kNaThreads, 0, st.stream>>>(static_cast<const double2*>(st.amps), st.dim(),
                                                                    tt, scratch);
    na_finish<<<1, kNaThreads, 0, st.stream>>>(scratch, (int)n_terms);
    count_launch(2);
    KB_CUDA(cudaGetLastError());
    double per[kMaxTerms];
    KB_CUDA(cudaMemcpyAsync(per, scratch + (size_t)kMaxTerms * kNaBlocks, sizeof(double) * n_terms,
                            cudaMemcpyDeviceToHost, st.stream));
    KB_CUDA(cudaStreamSynchronize(st.stream));
    double total = 0.0;  // coefficient-weighted, in term order (observable.cpp:85-91)
    for (uint64_t t = 0; t < n_terms; ++t) total += coeffs[t] * per[t];
    *out = total;
    return KETGPU_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return KETGPU_ERR_LOGIC;
  }
}
