// gates.cu -- per-gate state-vector kernels and the SIMT dense-block apply.
//
// Replaces the CPU loops of ket's src/simulator.cpp:
//   apply_single / rotations / U       :23-97   -> pair_kernel (general 2x2)
//   apply_cx / apply_ccx / apply_swap /
//   apply_cswap                        :99-109, 204-242 -> pair_kernel (swap)
//   apply_cy / apply_ch / controlled   :112-200 -> pair_kernel (general, controls
//                                                  fixed to 1)
//   apply_cphase (CZ, CP), diagonal 1q :246-254 -> phase_kernel
//   apply_matrix                       :357-393 -> fused_simt_kernel
// The reference scans all 2^n indices with a mask test per index; here every
// thread is handed an owner index directly: the pair (or phase) index i is
// spread into the 2^n index space by inserting zero bits at the fixed qubit
// positions, so only the amplitudes a gate changes are read and written.
#include <cuda_runtime.h>

#include <cstdint>

#include "internal.h"

namespace kb {
namespace {

template <typename R>
struct C2;
template <>
struct C2<float> {
  using T = float2;
};
template <>
struct C2<double> {
  using T = double2;
};

template <typename R>
struct Mat2 {
  R re[4], im[4];
};

// Insert a zero bit at each fixed position (ascending), as the reference
// spreads its outer index (simulator.cpp:379-382).
__device__ __forceinline__ uint64_t spread(uint64_t i, const int* fixed, int nfixed) {
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    if (j < nfixed) {
      const int f = fixed[j];
      i = ((i >> f) << (f + 1)) | (i & ((uint64_t{1} << f) - 1));
    }
  }
  return i;
}

struct PairGeom {
  uint64_t count;
  uint64_t p0, p1;
  int fixed[3];
  int nfixed;
};

constexpr int kUnroll = 4;
constexpr int kThreads = 256;

template <typename R, int MODE>
__global__ void __launch_bounds__(kThreads)
    pair_kernel(typename C2<R>::T* __restrict__ s, PairGeom g, Mat2<R> m) {
  using T = typename C2<R>::T;
  const uint64_t start = (uint64_t)blockIdx.x * (kThreads * kUnroll) + threadIdx.x;
  T a[kUnroll], b[kUnroll];
  uint64_t k0[kUnroll];
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) {
    const uint64_t i = start + (uint64_t)u * kThreads;
    k0[u] = ~uint64_t{0};
    if (i < g.count) {
      const uint64_t base = spread(i, g.fixed, g.nfixed);
      k0[u] = base;
      a[u] = s[base | g.p0];
      b[u] = s[base | g.p1];
    }
  }
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) {
    if (k0[u] == ~uint64_t{0}) continue;
    T x, y;
    if (MODE == kPairSwap) {
      x = b[u];
      y = a[u];
    } else if (MODE == kPairDiag) {
      x.x = m.re[0] * a[u].x - m.im[0] * a[u].y;
      x.y = m.re[0] * a[u].y + m.im[0] * a[u].x;
      y.x = m.re[3] * b[u].x - m.im[3] * b[u].y;
      y.y = m.re[3] * b[u].y + m.im[3] * b[u].x;
    } else {
      x.x = m.re[0] * a[u].x - m.im[0] * a[u].y + m.re[1] * b[u].x - m.im[1] * b[u].y;
      x.y = m.re[0] * a[u].y + m.im[0] * a[u].x + m.re[1] * b[u].y + m.im[1] * b[u].x;
      y.x = m.re[2] * a[u].x - m.im[2] * a[u].y + m.re[3] * b[u].x - m.im[3] * b[u].y;
      y.y = m.re[2] * a[u].y + m.im[2] * a[u].x + m.re[3] * b[u].y + m.im[3] * b[u].x;
    }
    s[k0[u] | g.p0] = x;
    s[k0[u] | g.p1] = y;
  }
}

template <typename R>
__global__ void __launch_bounds__(kThreads)
    phase_kernel(typename C2<R>::T* __restrict__ s, PairGeom g, R pre, R pim) {
  using T = typename C2<R>::T;
  const uint64_t start = (uint64_t)blockIdx.x * (kThreads * kUnroll) + threadIdx.x;
  T a[kUnroll];
  uint64_t k[kUnroll];
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) {
    const uint64_t i = start + (uint64_t)u * kThreads;
    k[u] = ~uint64_t{0};
    if (i < g.count) {
      k[u] = spread(i, g.fixed, g.nfixed) | g.p0;
      a[u] = s[k[u]];
    }
  }
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) {
    if (k[u] == ~uint64_t{0}) continue;
    T x;
    x.x = pre * a[u].x - pim * a[u].y;
    x.y = pre * a[u].y + pim * a[u].x;
    s[k[u]] = x;
  }
}

// ---------------------------------------------------------------------------
// Vectorised complex64 forms.  When no fixed qubit is qubit 0, pair indices
// 2t and 2t+1 own adjacent amplitudes, so one 16-byte load carries two
// complex64 values per side of the pair; a 1-qubit gate on qubit 0 owns the
// adjacent amplitudes (2i, 2i+1) themselves.

__device__ __forceinline__ float2 cmul_add(float ar, float ai, float2 a, float br, float bi, float2 b) {
  return make_float2(ar * a.x - ai * a.y + br * b.x - bi * b.y, ar * a.y + ai * a.x + br * b.y + bi * b.x);
}

template <int MODE>
__device__ __forceinline__ void pair_update(const Mat2<float>& m, float2 a, float2 b, float2& x, float2& y) {
  if (MODE == kPairSwap) {
    x = b;
    y = a;
  } else if (MODE == kPairDiag) {
    x = make_float2(m.re[0] * a.x - m.im[0] * a.y, m.re[0] * a.y + m.im[0] * a.x);
    y = make_float2(m.re[3] * b.x - m.im[3] * b.y, m.re[3] * b.y + m.im[3] * b.x);
  } else {
    x = cmul_add(m.re[0], m.im[0], a, m.re[1], m.im[1], b);
    y = cmul_add(m.re[2], m.im[2], a, m.re[3], m.im[3], b);
  }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads)
    pair_kernel_v2(float2* __restrict__ s, PairGeom g, Mat2<float> m) {
  const uint64_t count2 = g.count >> 1;
  const uint64_t start = (uint64_t)blockIdx.x * (kThreads * kUnroll) + threadIdx.x;
  float4 a[kUnroll], b[kUnroll];
  uint64_t k0[kUnroll];
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) {
    const uint64_t t = start + (uint64_t)u * kThreads;
    k0[u] = ~uint64_t{0};
    if (t < count2) {
      k0[u] = spread(2 * t, g.fixed, g.nfixed);
      a[u] = *reinterpret_cast<const float4*>(s + (k0[u] | g.p0));
      b[u] = *reinterpret_cast<const float4*>(s + (k0[u] | g.p1));
    }
  }
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) {
    if (k0[u] == ~uint64_t{0}) continue;
    float2 x0, y0, x1, y1;
    pair_update<MODE>(m, make_float2(a[u].x, a[u].y), make_float2(b[u].x, b[u].y), x0, y0);
    pair_update<MODE>(m, make_float2(a[u].z, a[u].w), make_float2(b[u].z, b[u].w), x1, y1);
    *reinterpret_cast<float4*>(s + (k0[u] | g.p0)) = make_float4(x0.x, x0.y, x1.x, x1.y);
    *reinterpret_cast<float4*>(s + (k0[u] | g.p1)) = make_float4(y0.x, y0.y, y1.x, y1.y);
  }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads)
    pair_kernel_q0(float2* __restrict__ s, uint64_t count, Mat2<float> m) {
  const uint64_t start = (uint64_t)blockIdx.x * (kThreads * kUnroll) + threadIdx.x;
  float4 v[kUnroll];
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) {
    const uint64_t i = start + (uint64_t)u * kThreads;
    if (i < count) v[u] = *reinterpret_cast<const float4*>(s + 2 * i);
  }
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) {
    const uint64_t i = start + (uint64_t)u * kThreads;
    if (i >= count) continue;
    float2 x, y;
    pair_update<MODE>(m, make_float2(v[u].x, v[u].y), make_float2(v[u].z, v[u].w), x, y);
    *reinterpret_cast<float4*>(s + 2 * i) = make_float4(x.x, x.y, y.x, y.y);
  }
}

__global__ void __launch_bounds__(kThreads)
    phase_kernel_v2(float2* __restrict__ s, PairGeom g, float pre, float pim) {
  const uint64_t count2 = g.count >> 1;
  const uint64_t start = (uint64_t)blockIdx.x * (kThreads * kUnroll) + threadIdx.x;
  float4 a[kUnroll];
  uint64_t k[kUnroll];
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) {
    const uint64_t t = start + (uint64_t)u * kThreads;
    k[u] = ~uint64_t{0};
    if (t < count2) {
      k[u] = spread(2 * t, g.fixed, g.nfixed) | g.p0;
      a[u] = *reinterpret_cast<const float4*>(s + k[u]);
    }
  }
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) {
    if (k[u] == ~uint64_t{0}) continue;
    const float4 x = a[u];
    *reinterpret_cast<float4*>(s + k[u]) = make_float4(pre * x.x - pim * x.y, pre * x.y + pim * x.x,
                                                       pre * x.z - pim * x.w, pre * x.w + pim * x.z);
  }
}

// ---------------------------------------------------------------------------
// Dense k-qubit block on CUDA cores (FP64 for complex128, FP32 for complex64
// when the tensor-core path is off).  A CTA owns a tile of 2^TB amplitudes:
// the k block qubits plus the lowest TB-k other qubits, so each of the 2^k
// target combinations is a contiguous run in memory.  The tile is staged in
// shared memory as [group][combination]; each thread computes 2048/256 = 8
// outputs out[g][r] = sum_c M[r][c] in[g][c]; the tile is written back in
// place with the same coalesced mapping.

constexpr int kTileBits = 11;

struct FusedGeom {
  int n, k, tb;           // tb = tile bits = min(kTileBits, n)
  int tile_pos[kTileBits];  // tile bit positions, ascending
  int is_target[kTileBits];
  uint64_t n_tiles;
};

template <typename R>
__global__ void __launch_bounds__(kThreads)
    fused_simt_kernel(typename C2<R>::T* __restrict__ s, FusedGeom g,
                      const typename C2<R>::T* __restrict__ mat_t) {
  using T = typename C2<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int dim = 1 << g.k;
  const int tile = 1 << g.tb;
  T* mt = reinterpret_cast<T*>(smem_raw);  // [c][r] : dim*dim
  T* buf = mt + dim * dim;                 // [group][comb] : tile
  __shared__ uint64_t off_lo[64], off_hi[64];
  __shared__ int idx_lo[64], idx_hi[64];

  for (int i = threadIdx.x; i < dim * dim; i += blockDim.x) mt[i] = mat_t[i];
  if (threadIdx.x < 128) {
    const int half = threadIdx.x >> 6, e = threadIdx.x & 63;
    uint64_t off = 0;
    int idx = 0, tcount = 0, gcount = 0;
    for (int j = 0; j < g.tb; ++j) {
      const bool t = g.is_target[j];
      const int sh = t ? tcount++ : (g.k + gcount++);
      const int local = j - 6 * half;
      if (local >= 0 && local < 6 && ((e >> local) & 1)) {
        off |= uint64_t{1} << g.tile_pos[j];
        idx |= 1 << sh;
      }
    }
    if (half == 0) {
      off_lo[e] = off;
      idx_lo[e] = idx;
    } else {
      off_hi[e] = off;
      idx_hi[e] = idx;
    }
  }
  __syncthreads();

  for (uint64_t t = blockIdx.x; t < g.n_tiles; t += gridDim.x) {
    // tile base: spread t over the non-tile positions
    uint64_t base = t;
    for (int j = 0; j < g.tb; ++j) {
      const int f = g.tile_pos[j];
      base = ((base >> f) << (f + 1)) | (base & ((uint64_t{1} << f) - 1));
    }
    for (int e = threadIdx.x; e < tile; e += blockDim.x) {
      const uint64_t off = off_lo[e & 63] + off_hi[e >> 6];
      buf[idx_lo[e & 63] + idx_hi[e >> 6]] = s[base + off];
    }
    __syncthreads();
    T out[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int o = threadIdx.x + j * kThreads;  // output index in [0, tile)
      if (o < tile) {
        const int r = o & (dim - 1);
        const T* in = buf + (o - r);
        R re = 0, im = 0;
        for (int c = 0; c < dim; ++c) {
          const T mv = mt[c * dim + r];
          const T x = in[c];
          re += mv.x * x.x - mv.y * x.y;
          im += mv.x * x.y + mv.y * x.x;
        }
        out[j].x = re;
        out[j].y = im;
      }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (threadIdx.x + j * kThreads < tile) buf[threadIdx.x + j * kThreads] = out[j];
    __syncthreads();
    for (int e = threadIdx.x; e < tile; e += blockDim.x) {
      const uint64_t off = off_lo[e & 63] + off_hi[e >> 6];
      s[base + off] = buf[idx_lo[e & 63] + idx_hi[e >> 6]];
    }
    __syncthreads();
  }
}

template <typename R>
__global__ void set_one_kernel(typename C2<R>::T* s) {
  typename C2<R>::T v;
  v.x = 1;
  v.y = 0;
  s[0] = v;
}

int sm_count(int device) {
  static int cached[64] = {0};
  if (device < 0 || device >= 64) return 148;
  if (!cached[device]) {
    int v = 0;
    KB_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device));
    cached[device] = v;
  }
  return cached[device];
}

template <typename R>
void launch_pair(const State& st, const Pass& p) {
  using T = typename C2<R>::T;
  PairGeom g{};
  g.nfixed = p.nfixed;
  for (int j = 0; j < 3; ++j) g.fixed[j] = p.fixed[j];
  g.count = st.dim() >> p.nfixed;
  g.p0 = p.p0;
  g.p1 = p.p1;
  T* s = static_cast<T*>(st.amps);
  // complex64: 16-byte forms when the layout allows them
  const bool vec2 = sizeof(R) == 4 && p.fixed[0] >= 1 && g.count >= 2;
  const bool q0 = sizeof(R) == 4 && p.kind == PassKind::Pair && p.nfixed == 1 && p.fixed[0] == 0;
  const uint64_t per_block = (uint64_t)kThreads * kUnroll;
  const uint64_t blocks = ((vec2 ? g.count / 2 : g.count) + per_block - 1) / per_block;
  Mat2<R> m;
  for (int j = 0; j < 4; ++j) {
    m.re[j] = (R)p.m[j].real();
    m.im[j] = (R)p.m[j].imag();
  }
  if (p.kind == PassKind::Phase) {
    if constexpr (sizeof(R) == 4) {
      if (vec2) {
        phase_kernel_v2<<<(unsigned)blocks, kThreads, 0, st.stream>>>(s, g, (float)p.m[0].real(),
                                                                      (float)p.m[0].imag());
        count_launch();
        KB_CUDA(cudaGetLastError());
        return;
      }
    }
    phase_kernel<R><<<(unsigned)blocks, kThreads, 0, st.stream>>>(s, g, (R)p.m[0].real(),
                                                                  (R)p.m[0].imag());
  } else {
    if constexpr (sizeof(R) == 4) {
      if (vec2 || q0) {
        if (vec2) {
          if (p.mode == kPairSwap)
            pair_kernel_v2<kPairSwap><<<(unsigned)blocks, kThreads, 0, st.stream>>>(s, g, m);
          else if (p.mode == kPairDiag)
            pair_kernel_v2<kPairDiag><<<(unsigned)blocks, kThreads, 0, st.stream>>>(s, g, m);
          else
            pair_kernel_v2<kPairGeneral><<<(unsigned)blocks, kThreads, 0, st.stream>>>(s, g, m);
        } else {
          if (p.mode == kPairSwap)
            pair_kernel_q0<kPairSwap><<<(unsigned)blocks, kThreads, 0, st.stream>>>(s, g.count, m);
          else if (p.mode == kPairDiag)
            pair_kernel_q0<kPairDiag><<<(unsigned)blocks, kThreads, 0, st.stream>>>(s, g.count, m);
          else
            pair_kernel_q0<kPairGeneral><<<(unsigned)blocks, kThreads, 0, st.stream>>>(s, g.count, m);
        }
        count_launch();
        KB_CUDA(cudaGetLastError());
        return;
      }
    }
    if (p.mode == kPairSwap)
      pair_kernel<R, kPairSwap><<<(unsigned)blocks, kThreads, 0, st.stream>>>(s, g, m);
    else if (p.mode == kPairDiag)
      pair_kernel<R, kPairDiag><<<(unsigned)blocks, kThreads, 0, st.stream>>>(s, g, m);
    else
      pair_kernel<R, kPairGeneral><<<(unsigned)blocks, kThreads, 0, st.stream>>>(s, g, m);
  }
  count_launch();
  KB_CUDA(cudaGetLastError());
}

template <typename R>
void launch_fused_simt(const State& st, const Pass& p, const void* mat_t) {
  using T = typename C2<R>::T;
  FusedGeom g{};
  g.n = st.n;
  g.k = p.k;
  g.tb = st.n < kTileBits ? st.n : kTileBits;
  // tile bits: the k targets plus the lowest non-target positions
  uint64_t tmask = 0;
  for (int b = 0; b < p.k; ++b) tmask |= uint64_t{1} << p.qubits[b];
  int extra = g.tb - p.k;
  uint64_t tiles_mask = tmask;
  for (int q = 0; q < st.n && extra > 0; ++q)
    if (!((tmask >> q) & 1)) {
      tiles_mask |= uint64_t{1} << q;
      --extra;
    }
  int j = 0;
  for (int q = 0; q < st.n; ++q)
    if ((tiles_mask >> q) & 1) {
      g.tile_pos[j] = q;
      g.is_target[j] = (int)((tmask >> q) & 1);
      ++j;
    }
  g.n_tiles = st.dim() >> g.tb;
  const int dim = 1 << p.k;
  const size_t smem = sizeof(T) * ((size_t)dim * dim + ((size_t)1 << g.tb));
  static bool attr_set[2] = {false, false};
  const int which = sizeof(R) == 8 ? 1 : 0;
  if (!attr_set[which]) {
    KB_CUDA(cudaFuncSetAttribute(fused_simt_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 200 * 1024));
    attr_set[which] = true;
  }
  uint64_t grid = (uint64_t)sm_count(st.device) * 4;
  if (grid > g.n_tiles) grid = g.n_tiles;
  fused_simt_kernel<R><<<(unsigned)grid, kThreads, smem, st.stream>>>(
      static_cast<T*>(st.amps), g, static_cast<const T*>(mat_t));
  count_launch();
  KB_CUDA(cudaGetLastError());
}


// ---------------------------------------------------------------------------
// Shared-memory runs (the plain method's staging of low-qubit gates).  A run
// of consecutive gates whose qubits all lie below kRunBits touches only
// amplitudes inside aligned chunks of 2^kRunBits; a CTA loads a chunk with
// coalesced 16-byte loads, applies each gate in turn in shared memory
// (exactly the pair / phase updates of the per-gate kernels, on chunk-local
// indices), and stores the chunk back: one HBM pass for the run instead of
// one per gate.

template <typename R>
struct RunGate {
  int32_t kind;  // 0 pair (mode below), 1 phase
  int32_t mode;  // kPairGeneral / kPairSwap / kPairDiag
  int32_t nfixed;
  int32_t fixed[3];
  uint32_t p0, p1;
  R re[4], im[4];
};

template <typename R>
__global__ void __launch_bounds__(kThreads)
    run_kernel(typename C2<R>::T* __restrict__ s, uint64_t n_chunks, int bits,
               const RunGate<R>* __restrict__ gates, int ngates) {
  using T = typename C2<R>::T;
  extern __shared__ __align__(16) unsigned char run_smem[];
  T* sm = reinterpret_cast<T*>(run_smem);
  RunGate<R>* sg = reinterpret_cast<RunGate<R>*>(run_smem + (sizeof(T) << kRunBits));
  for (int i = threadIdx.x; i < ngates; i += kThreads) sg[i] = gates[i];
  const int size = 1 << bits;
  constexpr int V = 16 / (int)sizeof(T);  // amplitudes per 16-byte word
  for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
    T* src = s + (c << bits);
    __syncthreads();
    for (int i = threadIdx.x; i < size / V; i += kThreads)
      reinterpret_cast<float4*>(sm)[i] = reinterpret_cast<const float4*>(src)[i];
    __syncthreads();
    for (int gi = 0; gi < ngates; ++gi) {
      const RunGate<R>& g = sg[gi];
      const int cnt = size >> g.nfixed;
      for (int i = threadIdx.x; i < cnt; i += kThreads) {
        const uint32_t base = (uint32_t)spread((uint64_t)i, g.fixed, g.nfixed);
        if (g.kind == 1) {
          const T a = sm[base | g.p0];
          T x;
          x.x = g.re[0] * a.x - g.im[0] * a.y;
          x.y = g.re[0] * a.y + g.im[0] * a.x;
          sm[base | g.p0] = x;
          continue;
        }
        const T a = sm[base | g.p0], b = sm[base | g.p1];
        T x, y;
        if (g.mode == kPairSwap) {
          x = b;
          y = a;
        } else if (g.mode == kPairDiag) {
          x.x = g.re[0] * a.x - g.im[0] * a.y;
          x.y = g.re[0] * a.y + g.im[0] * a.x;
          y.x = g.re[3] * b.x - g.im[3] * b.y;
          y.y = g.re[3] * b.y + g.im[3] * b.x;
        } else {
          x.x = g.re[0] * a.x - g.im[0] * a.y + g.re[1] * b.x - g.im[1] * b.y;
          x.y = g.re[0] * a.y + g.im[0] * a.x + g.re[1] * b.y + g.im[1] * b.x;
          y.x = g.re[2] * a.x - g.im[2] * a.y + g.re[3] * b.x - g.im[3] * b.y;
          y.y = g.re[2] * a.y + g.im[2] * a.x + g.re[3] * b.y + g.im[3] * b.x;
        }
        sm[base | g.p0] = x;
        sm[base | g.p1] = y;
      }
      __syncthreads();
    }
    for (int i = threadIdx.x; i < size / V; i += kThreads)
      reinterpret_cast<float4*>(src)[i] = reinterpret_cast<const float4*>(sm)[i];
  }
}

template <typename R>
void append_run_gates(const std::vector<Pass>& gates, std::vector<unsigned char>& out) {
  for (const Pass& p : gates) {
    RunGate<R> g{};
    g.kind = p.kind == PassKind::Phase ? 1 : 0;
    g.mode = p.mode;
    g.nfixed = p.nfixed;
    for (int j = 0; j < 3; ++j) g.fixed[j] = p.fixed[j];
    g.p0 = (uint32_t)p.p0;
    g.p1 = (uint32_t)p.p1;
    for (int j = 0; j < 4; ++j) {
      g.re[j] = (R)p.m[j].real();
      g.im[j] = (R)p.m[j].imag();
    }
    const unsigned char* b = reinterpret_cast<const unsigned char*>(&g);
    out.insert(out.end(), b, b + sizeof g);
  }
}

}  // namespace

void run_device_data(const std::vector<Pass>& gates, int precision, std::vector<unsigned char>& out) {
  out.clear();
  if (precision == KETGPU_C64) append_run_gates<float>(gates, out);
  else append_run_gates<double>(gates, out);
}

void launch_run(const State& st, const Pass& p, const void* data) {
  const int bits = st.n < kRunBits ? st.n : kRunBits;
  const uint64_t n_chunks = st.dim() >> bits;
  static int sms[64] = {0};
  if (!sms[st.device]) sms[st.device] = sm_count(st.device);
  uint64_t grid = (uint64_t)sms[st.device] * 8;
  if (grid > n_chunks) grid = n_chunks;
  if (st.precision == KETGPU_C64) {
    const size_t smem = (sizeof(float2) << kRunBits) + sizeof(RunGate<float>) * (size_t)p.n_gates;
    run_kernel<float><<<(unsigned)grid, kThreads, smem, st.stream>>>(
        static_cast<float2*>(st.amps), n_chunks, bits, static_cast<const RunGate<float>*>(data), p.n_gates);
  } else {
    const size_t smem = (sizeof(double2) << kRunBits) + sizeof(RunGate<double>) * (size_t)p.n_gates;
    static bool attr[64] = {false};
    if (!attr[st.device]) {
      KB_CUDA(cudaFuncSetAttribute(run_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)((sizeof(double2) << kRunBits) + sizeof(RunGate<double>) * kRunMaxGates)));
      attr[st.device] = true;
    }
    run_kernel<double><<<(unsigned)grid, kThreads, smem, st.stream>>>(
        static_cast<double2*>(st.amps), n_chunks, bits, static_cast<const RunGate<double>*>(data), p.n_gates);
  }
  count_launch();
  KB_CUDA(cudaGetLastError());
}

double Pass::bytes(int n, size_t amp) const {
  const double dim = (double)(uint64_t{1} << n);
  if (kind == PassKind::Fused || kind == PassKind::Diagonal || kind == PassKind::SharedRun) return 2.0 * amp * dim;
  if (kind == PassKind::NormCapture) return amp * dim;
  // the norm read (unless the block before summed it) plus the rescale
  if (kind == PassKind::NormRestore) return (norm_out ? 2.0 : 3.0) * amp * dim;
  if (kind == PassKind::Phase) return 2.0 * amp * dim / (double)(uint64_t{1} << nfixed);
  // pair: two amplitudes per pair, both read and written
  return 2.0 * amp * 2.0 * dim / (double)(uint64_t{1} << nfixed);
}

__global__ void store_one_kernel(double* p) { *p = 1.0; }

void set_ground(const State& s) {
  s.touch();
  s.ground_version = s.version;
  KB_CUDA(cudaMemsetAsync(s.amps, 0, s.dim() * s.amp_bytes(), s.stream));
  if (s.precision == KETGPU_C64)
    set_one_kernel<float><<<1, 1, 0, s.stream>>>(static_cast<float2*>(s.amps));
  else
    set_one_kernel<double><<<1, 1, 0, s.stream>>>(static_cast<double2*>(s.amps));
  count_launch();
  KB_CUDA(cudaGetLastError());
}

void launch_pass(const State& s, const Plan& plan, const Pass& p) {
  const bool ground = s.version == s.ground_version;
  s.touch();
  if (p.kind == PassKind::NormCapture) {
    if (ground) {  // |0...0>: the squared norm is 1, no pass over the state
      store_one_kernel<<<1, 1, 0, s.stream>>>(plan.d_norm);
      count_launch();
      KB_CUDA(cudaGetLastError());
    } else {
      norm_to_device(s, plan.d_norm + 2, plan.d_norm);
    }
    return;
  }
  if (p.kind == PassKind::NormRestore) {
    if (p.norm_out)  // the block before summed |out|^2 per CTA into the partials
      norm_from_partials(s, plan.d_norm + 2, plan.d_norm + 1);
    else
      norm_to_device(s, plan.d_norm + 2, plan.d_norm + 1);
    rescale_state(s, plan.d_norm, plan.d_norm + 1);
    return;
  }
  if (p.kind == PassKind::Diagonal) {
    launch_diag(s, p, static_cast<const char*>(plan.d_diag) + plan.offdiag[p.diag_index]);
    return;
  }
  if (p.kind == PassKind::SharedRun) {
    launch_run(s, p, static_cast<const char*>(plan.d_runs) + plan.offrun[p.run_index]);
    return;
  }
  if (p.kind != PassKind::Fused) {
    if (s.precision == KETGPU_C64)
      launch_pair<float>(s, p);
    else
      launch_pair<double>(s, p);
    return;
  }
  if (s.precision == KETGPU_C128) {
    launch_fused_simt<double>(s, p, static_cast<const char*>(plan.d_mat64) + plan.off64[p.mat_index]);
  } else if (p.tensor) {
    launch_fused_tc(s, p, static_cast<const char*>(plan.d_tc) + plan.offtc[p.mat_index],
                    p.norm_out ? plan.d_norm + 2 : nullptr);
  } else {
    launch_fused_simt<float>(s, p, static_cast<const char*>(plan.d_mat32) + plan.off32[p.mat_index]);
  }
}

}  // namespace kb
