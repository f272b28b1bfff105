// adjoint.cu -- reverse-sweep (adjoint) gradients of <psi(theta)|H|psi(theta)>
// for a batch of parameter sets, H a Pauli sum.
//
// No ket counterpart: ket evaluates ket::expval(run(circuit), PauliSum)
// (src/observable.cpp:85-91) and has no derivatives.  The algebra follows
// ket's gate matrices (src/simulator.cpp:73-89 for Rx/Ry/Rz, :166-189 for the
// controlled rotations, :322-324 for CP) and Pauli actions
// (src/observable.cpp:68-118):
//   forward   psi_N = U_N ... U_1 |0>, checkpoints at layer boundaries
//   lambda    lambda = H psi_N,   <H> = Re <psi_N|lambda>
//   reverse   for i = N..1:  g_i = Im <lambda|G_i|psi_i>  (U_i = exp(-i t G_i / 2))
//                            psi <- U_i^dag psi, lambda <- U_i^dag lambda
// For CP(t) = diag(1,1,1,e^{it}) the term is -2 Im <lambda|P11|psi>.
// One kernel per gate does the inner-product partial sums (FP64) and the two
// inverse applications in a single pass over psi and lambda; all parameter
// sets of a chunk share every launch (gridDim.y = set).  Layers are the
// barrier-delimited runs of ops; with checkpoint_every = m the forward state
// is stored every m layers and the reverse sweep restarts psi from it, so
// the uncomputation error does not accumulate across segments.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <cstdio>
#include <map>
#include <mutex>
#include <cmath>
#include <cstring>
#include <memory>
#include <queue>
#include <string>
#include <utility>
#include <vector>

#include "internal.h"
#include "adj_tile.cuh"

#define KB_API extern "C" __attribute__((visibility("default")))

namespace kb {
State* create_state(int n, int precision);
void destroy_state(State* s);

namespace {

template <typename R>
struct C2T;
template <>
struct C2T<float> {
  using T = float2;
};
template <>
struct C2T<double> {
  using T = double2;
};

constexpr int kAThreads = 256;

struct GateGeom {
  uint64_t count;  // pairs (or phase elements) per state
  uint64_t p0, p1;
  int fixed[3];
  int nfixed;
  int kind;   // 0 pair general, 1 pair swap, 2 phase
  int gen;    // generator for the gradient: 0 none, 1 X, 2 Y, 3 Z, 4 P11 (phase)
  int pslot;  // gradient slot (parameter index) or -1
};

__device__ __forceinline__ uint64_t spread3(uint64_t i, const int* fixed, int nfixed) {
#pragma unroll
  for (int j = 0; j < 3; ++j)
    if (j < nfixed) {
      const int f = fixed[j];
      i = ((i >> f) << (f + 1)) | (i & ((uint64_t{1} << f) - 1));
    }
  return i;
}

// Forward application of one gate to every state of the chunk: mats holds a
// 2x2 (or the phase in slot 0) per state, FP64 interleaved.
template <typename R>
__global__ void fwd_gate(typename C2T<R>::T* __restrict__ states, uint64_t dim, GateGeom g,
                         const double* __restrict__ mats) {
  using T = typename C2T<R>::T;
  T* s = states + (uint64_t)blockIdx.y * dim;
  const double* m = mats + (size_t)blockIdx.y * 8;
  const R m0r = (R)m[0], m0i = (R)m[1], m1r = (R)m[2], m1i = (R)m[3];
  const R m2r = (R)m[4], m2i = (R)m[5], m3r = (R)m[6], m3i = (R)m[7];
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = spread3(i, g.fixed, g.nfixed);
    if (g.kind == 2) {
      const T a = s[b | g.p0];
      T r;
      r.x = m0r * a.x - m0i * a.y;
      r.y = m0r * a.y + m0i * a.x;
      s[b | g.p0] = r;
      continue;
    }
    const T a = s[b | g.p0], c = s[b | g.p1];
    if (g.kind == 1) {
      s[b | g.p0] = c;
      s[b | g.p1] = a;
      continue;
    }
    T x, y;
    x.x = m0r * a.x - m0i * a.y + m1r * c.x - m1i * c.y;
    x.y = m0r * a.y + m0i * a.x + m1r * c.y + m1i * c.x;
    y.x = m2r * a.x - m2i * a.y + m3r * c.x - m3i * c.y;
    y.y = m2r * a.y + m2i * a.x + m3r * c.y + m3i * c.x;
    s[b | g.p0] = x;
    s[b | g.p1] = y;
  }
}

// Reverse step: partial Im <lambda|G|psi> (FP64) for this gate, then
// psi <- U^dag psi and lambda <- U^dag lambda.  mats holds U (not U^dag).
template <typename R>
__global__ void __launch_bounds__(kAThreads)
    rev_gate(typename C2T<R>::T* __restrict__ psi, typename C2T<R>::T* __restrict__ lam, uint64_t dim, GateGeom g,
             const double* __restrict__ mats, double* __restrict__ partial /* [set][blocks] */) {
  using T = typename C2T<R>::T;
  __shared__ double sh[32];
  T* s = psi + (uint64_t)blockIdx.y * dim;
  T* l = lam + (uint64_t)blockIdx.y * dim;
  const double* m = mats + (size_t)blockIdx.y * 8;
  // U^dag entries
  const R d0r = (R)m[0], d0i = (R)-m[1], d1r = (R)m[4], d1i = (R)-m[5];
  const R d2r = (R)m[2], d2i = (R)-m[3], d3r = (R)m[6], d3i = (R)-m[7];
  double acc = 0.0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < g.count;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = spread3(i, g.fixed, g.nfixed);
    if (g.kind == 2) {
      const T a = s[b | g.p0], lv = l[b | g.p0];
      if (g.gen == 4) acc += (double)lv.x * (double)a.y - (double)lv.y * (double)a.x;  // Im(conj(l) a)
      T r, q;
      r.x = d0r * a.x - d0i * a.y;
      r.y = d0r * a.y + d0i * a.x;
      q.x = d0r * lv.x - d0i * lv.y;
      q.y = d0r * lv.y + d0i * lv.x;
      s[b | g.p0] = r;
      l[b | g.p0] = q;
      continue;
    }
    const T a0 = s[b | g.p0], a1 = s[b | g.p1];
    const T l0 = l[b | g.p0], l1 = l[b | g.p1];
    if (g.gen) {
      // G psi restricted to the pair
      double g0r, g0i, g1r, g1i;
      if (g.gen == 1) {  // X
        g0r = a1.x; g0i = a1.y; g1r = a0.x; g1i = a0.y;
      } else if (g.gen == 2) {  // Y: (-i a1, i a0)
        g0r = a1.y; g0i = -(double)a1.x; g1r = -(double)a0.y; g1i = a0.x;
      } else {  // Z
        g0r = a0.x; g0i = a0.y; g1r = -(double)a1.x; g1i = -(double)a1.y;
      }
      // Im(conj(l0) g0 + conj(l1) g1)
      acc += (double)l0.x * g0i - (double)l0.y * g0r + (double)l1.x * g1i - (double)l1.y * g1r;
    }
    if (g.kind == 1) {
      s[b | g.p0] = a1;
      s[b | g.p1] = a0;
      l[b | g.p0] = l1;
      l[b | g.p1] = l0;
      continue;
    }
    T x, y;
    x.x = d0r * a0.x - d0i * a0.y + d1r * a1.x - d1i * a1.y;
    x.y = d0r * a0.y + d0i * a0.x + d1r * a1.y + d1i * a1.x;
    y.x = d2r * a0.x - d2i * a0.y + d3r * a1.x - d3i * a1.y;
    y.y = d2r * a0.y + d2i * a0.x + d3r * a1.y + d3i * a1.x;
    s[b | g.p0] = x;
    s[b | g.p1] = y;
    x.x = d0r * l0.x - d0i * l0.y + d1r * l1.x - d1i * l1.y;
    x.y = d0r * l0.y + d0i * l0.x + d1r * l1.y + d1i * l1.x;
    y.x = d2r * l0.x - d2i * l0.y + d3r * l1.x - d3i * l1.y;
    y.y = d2r * l0.y + d2i * l0.x + d3r * l1.y + d3i * l1.x;
    l[b | g.p0] = x;
    l[b | g.p1] = y;
  }
  if (g.gen == 0) return;
  // fixed-order block reduction
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) sh[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    partial[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = t;
  }
}

// lambda = H psi for every state of the chunk (FP64 accumulation per
// amplitude), and per-block partials of Re <psi|lambda>.
template <typename R>
__global__ void __launch_bounds__(kAThreads)
    ham_apply(const typename C2T<R>::T* __restrict__ psi, typename C2T<R>::T* __restrict__ lam, uint64_t dim,
              const uint64_t* __restrict__ flips, const uint64_t* __restrict__ signs, const int* __restrict__ qs,
              const double* __restrict__ coeffs, int nterms, double* __restrict__ partial) {
  using T = typename C2T<R>::T;
  __shared__ double sh[32];
  const T* s = psi + (uint64_t)blockIdx.y * dim;
  T* l = lam + (uint64_t)blockIdx.y * dim;
  double e = 0.0;
  for (uint64_t y = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; y < dim;
       y += (uint64_t)gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int t = 0; t < nterms; ++t) {
      const uint64_t x = y ^ flips[t];
      const T a = s[x];
      // phase i^q times (-1)^popcount(x & sign)
      double ar = a.x, ai = a.y, vr, vi;
      switch (qs[t]) {
        case 0: vr = ar; vi = ai; break;
        case 1: vr = -ai; vi = ar; break;
        case 2: vr = -ar; vi = -ai; break;
        default: vr = ai; vi = -ar; break;
      }
      const double c = (__popcll(x & signs[t]) & 1) ? -coeffs[t] : coeffs[t];
      re += c * vr;
      im += c * vi;
    }
    T out;
    out.x = (R)re;
    out.y = (R)im;
    l[y] = out;
    const T p = s[y];
    e += (double)p.x * re + (double)p.y * im;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
  if (lane == 0) sh[warp] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    partial[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = t;
  }
}

// lambda = H psi for states larger than L2, split by the top qubit.  A
// Pauli term maps output half h to source half h ^ (flip's top bit), so the
// terms are grouped by that bit and each output half is built in two passes:
// first from the terms that read the same half, then (adding to lambda) from
// those that read the other half.  Each pass gathers from one half (67 MB at
// 24 qubits, complex64), which stays in L2 while the pass's terms revisit
// it.  The grid (CTAs per set x sets) covers about one set at a time.  Terms
// sit in shared memory with the phase i^q folded into a complex
// coefficient; eight gathers are in flight per thread.  The last pass of a
// half adds Re <psi|lambda> over it into per-CTA partials.
constexpr int kHamSmemTerms = 1024;
struct HamTerm {
  uint64_t flip, sign;
  double cr, ci;
};

template <typename R>
__global__ void __launch_bounds__(kAThreads)
    ham_half(const typename C2T<R>::T* __restrict__ psi, typename C2T<R>::T* __restrict__ lam, uint64_t dim, int h,
             int first, int last, const HamTerm* __restrict__ terms, int nterms, double* __restrict__ epart) {
  using T = typename C2T<R>::T;
  __shared__ double sh[32];
  extern __shared__ __align__(16) unsigned char hsm[];
  HamTerm* st = reinterpret_cast<HamTerm*>(hsm);
  for (int i = threadIdx.x; i < nterms; i += blockDim.x) st[i] = terms[i];
  __syncthreads();
  const T* s = psi + (uint64_t)blockIdx.y * dim;
  T* l = lam + (uint64_t)blockIdx.y * dim;
  const uint64_t half = dim >> 1, lo = h ? half : 0, hi = h ? dim : half;
  double e = 0.0;
  for (uint64_t y = lo + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; y < hi;
       y += (uint64_t)gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    if (!first) {  // lambda and psi[y] stream through (evict-first) so the
                   // gathered half keeps L2
      const T p = __ldcs(l + y);
      re = p.x;
      im = p.y;
    }
    int t = 0;
    for (; t + 8 <= nterms; t += 8) {
      T a[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) a[u] = s[y ^ st[t + u].flip];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const HamTerm& hm = st[t + u];
        const double ar = a[u].x, ai = a[u].y;
        const bool neg = __popcll((y ^ hm.flip) & hm.sign) & 1;
        const double cr = neg ? -hm.cr : hm.cr, ci = neg ? -hm.ci : hm.ci;
        re += cr * ar - ci * ai;
        im += cr * ai + ci * ar;
      }
    }
    for (; t < nterms; ++t) {
      const HamTerm& hm = st[t];
      const T a = s[y ^ hm.flip];
      const double ar = a.x, ai = a.y;
      const bool neg = __popcll((y ^ hm.flip) & hm.sign) & 1;
      const double cr = neg ? -hm.cr : hm.cr, ci = neg ? -hm.ci : hm.ci;
      re += cr * ar - ci * ai;
      im += cr * ai + ci * ar;
    }
    T out;
    out.x = (R)re;
    out.y = (R)im;
    __stcs(l + y, out);
    if (last) {
      const T p = __ldcs(s + y);
      e += (double)p.x * re + (double)p.y * im;
    }
  }
  if (!last) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
  if (lane == 0) sh[warp] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += sh[w];
    epart[((size_t)blockIdx.y * 2 + h) * gridDim.x + blockIdx.x] += v;
  }
}

template <typename R>
__global__ void ground_batch(typename C2T<R>::T* states, uint64_t dim) {
  typename C2T<R>::T one;
  one.x = 1;
  one.y = 0;
  states[(uint64_t)blockIdx.x * dim] = one;
}


// ---------------------------------------------------------------------------
// Tiled sweeps.  The per-gate kernels above stream psi (and lambda) through
// HBM once per gate.  The tiled form groups consecutive gates into blocks
// whose qubits fit one tile of TB qubits (always including qubits 0-4, so a
// warp's 32 consecutive tile elements are 32 consecutive amplitudes), loads
// each tile of psi and lambda into shared memory once, and runs the whole
// block there: the forward applications, or in the reverse sweep the
// gradient inner products and the inverse applications of every gate of the
// block.  Inside a block, gates are run in phases: a phase names RB tile bits
// that each thread holds in registers (2^RB amplitudes of each state), so
// every gate whose target bits are among them is register arithmetic; a
// diagonal gate needs no register bits at all.  Gradient partial sums are
// formed per thread over its pairs in the state's precision, reduced across
// the warp in FP64 and accumulated per warp and gate in shared memory (FP64),
// then summed in fixed order over warps, CTAs and (on the host) blocks.

// TileCfg, TGate, TPhase, TileGeom, the swizzle, the asynchronous copy and
// the packed complex64 gate code live in adj_tile.cuh, shared with the
// per-block kernels compiled at run time.
using namespace kbt;

template <typename R>
struct CM2 {
  R r[4], i[4];
};

// m (U, row-major, 8 values re/im interleaved) or its conjugate transpose.
template <typename R, bool DAG>
__device__ __forceinline__ CM2<R> load_cm2(const R* m) {
  CM2<R> c;
  if (!DAG) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      c.r[k] = m[2 * k];
      c.i[k] = m[2 * k + 1];
    }
  } else {
    c.r[0] = m[0], c.i[0] = -m[1];
    c.r[1] = m[4], c.i[1] = -m[5];
    c.r[2] = m[2], c.i[2] = -m[3];
    c.r[3] = m[6], c.i[3] = -m[7];
  }
  return c;
}

template <typename T, typename R>
__device__ __forceinline__ void mul2(const CM2<R>& c, T& a, T& b) {
  T x, y;
  x.x = c.r[0] * a.x - c.i[0] * a.y + c.r[1] * b.x - c.i[1] * b.y;
  x.y = c.r[0] * a.y + c.i[0] * a.x + c.r[1] * b.y + c.i[1] * b.x;
  y.x = c.r[2] * a.x - c.i[2] * a.y + c.r[3] * b.x - c.i[3] * b.y;
  y.y = c.r[2] * a.y + c.i[2] * a.x + c.r[3] * b.y + c.i[3] * b.x;
  a = x;
  b = y;
}

template <typename T, typename R>
__device__ __forceinline__ void mul2_real(const CM2<R>& c, T& a, T& b) {
  T x, y;
  x.x = c.r[0] * a.x + c.r[1] * b.x;
  x.y = c.r[0] * a.y + c.r[1] * b.y;
  y.x = c.r[2] * a.x + c.r[3] * b.x;
  y.y = c.r[2] * a.y + c.r[3] * b.y;
  a = x;
  b = y;
}

template <typename T, typename R>
__device__ __forceinline__ void cmul(T& a, R pr, R pi) {
  const R x = pr * a.x - pi * a.y;
  a.y = pr * a.y + pi * a.x;
  a.x = x;
}

template <typename T, typename R>
__device__ __forceinline__ void tswap(T& a, T& b) {
  const T t = a;
  a = b;
  b = t;
}

// Im <l|G|a> on one pair for the generators X (1), Y (2), Z (3).
template <typename T, typename R>
__device__ __forceinline__ R pair_grad(int gen, const T& a0, const T& a1, const T& l0, const T& l1) {
  if (gen == 1) return (l0.x * a1.y - l0.y * a1.x) + (l1.x * a0.y - l1.y * a0.x);
  if (gen == 2) return (l1.x * a0.x + l1.y * a0.y) - (l0.x * a1.x + l0.y * a1.y);
  return (l0.x * a0.y - l0.y * a0.x) - (l1.x * a1.y - l1.y * a1.x);
}

// Gate bodies.  A thread holds the 2^RB register elements j of its group; S
// (A, B) are register slots known at compile time; RC says whether some
// control bits are register bits (then each j is tested against cm_r).
// Forward (REV = false) applies U to p; reverse adds the gradient term and
// applies U^dag to p and q.

template <typename R, int RB, int S, bool REV, bool RC>
__device__ __forceinline__ R tile_pair(typename C2T<R>::T* p, typename C2T<R>::T* q, const TGate& g,
                                       const R* m) {
  R part = 0;
  if constexpr (S < RB) {
    if (g.kind == kTPairSwap) {
#pragma unroll
      for (int j = 0; j < (1 << RB); ++j) {
        if (j & (1 << S)) continue;
        if (RC && (j & g.cm_r) != g.cm_r) continue;
        tswap<typename C2T<R>::T, R>(p[j], p[j | (1 << S)]);
        if (REV) tswap<typename C2T<R>::T, R>(q[j], q[j | (1 << S)]);
      }
      return part;
    }
    const CM2<R> c = load_cm2<R, REV>(m);
    const bool real = g.real;
    const int gen = REV ? g.gen : 0;
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
      if (j & (1 << S)) continue;
      const int j1 = j | (1 << S);
      if (RC && (j & g.cm_r) != g.cm_r) continue;
      if (REV && gen) part += pair_grad<typename C2T<R>::T, R>(gen, p[j], p[j1], q[j], q[j1]);
      if (real) {
        mul2_real(c, p[j], p[j1]);
        if (REV) mul2_real(c, q[j], q[j1]);
      } else {
        mul2(c, p[j], p[j1]);
        if (REV) mul2(c, q[j], q[j1]);
      }
    }
  }
  return part;
}

template <typename R, int RB, int A, int B, bool REV, bool RC>
__device__ __forceinline__ void tile_swap2(typename C2T<R>::T* p, typename C2T<R>::T* q, const TGate& g) {
  if constexpr (A < RB && B < RB && A < B) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
      if (!(j & (1 << A)) || (j & (1 << B))) continue;
      if (RC && (j & g.cm_r) != g.cm_r) continue;
      const int j1 = j ^ (1 << A) ^ (1 << B);
      tswap<typename C2T<R>::T, R>(p[j], p[j1]);
      if (REV) tswap<typename C2T<R>::T, R>(q[j], q[j1]);
    }
  }
}

// Diagonal gate whose target is register slot S: diag(m0, m3).
template <typename R, int RB, int S, bool REV, bool RC>
__device__ __forceinline__ R tile_diag_reg(typename C2T<R>::T* p, typename C2T<R>::T* q, const TGate& g,
                                           const R* m) {
  R part = 0;
  if constexpr (S < RB) {
    const R m0r = m[0], m0i = REV ? -m[1] : m[1], m3r = m[6], m3i = REV ? -m[7] : m[7];
    const int gen = REV ? g.gen : 0;
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
      if (RC && (j & g.cm_r) != g.cm_r) continue;
      const bool bit = (j >> S) & 1;
      if (REV && gen) {
        const R im = q[j].x * p[j].y - q[j].y * p[j].x;  // Im(conj(l) a)
        if (gen == 3) part += bit ? -im : im;
        else if (bit) part += im;  // P11
      }
      cmul(p[j], bit ? m3r : m0r, bit ? m3i : m0i);
      if (REV) cmul(q[j], bit ? m3r : m0r, bit ? m3i : m0i);
    }
  }
  return part;
}

// Diagonal gate whose target is a group bit: one phase for all of the
// thread's elements.
template <typename R, int RB, bool REV, bool RC>
__device__ __forceinline__ R tile_diag_grp(typename C2T<R>::T* p, typename C2T<R>::T* q, const TGate& g,
                                           const R* m, bool bit) {
  R part = 0;
  const R pr = bit ? m[6] : m[0];
  const R pi = REV ? -(bit ? m[7] : m[1]) : (bit ? m[7] : m[1]);
  const int gen = REV ? g.gen : 0;
#pragma unroll
  for (int j = 0; j < (1 << RB); ++j) {
    if (RC && (j & g.cm_r) != g.cm_r) continue;
    if (REV && gen) part += q[j].x * p[j].y - q[j].y * p[j].x;
    cmul(p[j], pr, pi);
    if (REV) cmul(q[j], pr, pi);
  }
  if (REV && gen) part = gen == 3 ? (bit ? -part : part) : (bit ? part : R(0));
  return part;
}

template <typename R, int RB, bool REV, bool RC>
__device__ __forceinline__ R tile_gate_rc(typename C2T<R>::T* p, typename C2T<R>::T* q, const TGate& g,
                                          const R* m, int gbase) {
  if (g.kind == kTDiag) {
    switch (g.tslot) {
      case 0: return tile_diag_reg<R, RB, 0, REV, RC>(p, q, g, m);
      case 1: return tile_diag_reg<R, RB, 1, REV, RC>(p, q, g, m);
      case 2: return tile_diag_reg<R, RB, 2, REV, RC>(p, q, g, m);
      case 3: return tile_diag_reg<R, RB, 3, REV, RC>(p, q, g, m);
      default: return tile_diag_grp<R, RB, REV, RC>(p, q, g, m, (gbase >> g.tbit) & 1);
    }
  }
  if (g.kind == kTSwap2) {
    switch (g.s0 * 4 + g.s1) {
      case 1: tile_swap2<R, RB, 0, 1, REV, RC>(p, q, g); break;
      case 2: tile_swap2<R, RB, 0, 2, REV, RC>(p, q, g); break;
      case 3: tile_swap2<R, RB, 0, 3, REV, RC>(p, q, g); break;
      case 6: tile_swap2<R, RB, 1, 2, REV, RC>(p, q, g); break;
      case 7: tile_swap2<R, RB, 1, 3, REV, RC>(p, q, g); break;
      case 11: tile_swap2<R, RB, 2, 3, REV, RC>(p, q, g); break;
      default: break;
    }
    return 0;
  }
  switch (g.s0) {
    case 0: return tile_pair<R, RB, 0, REV, RC>(p, q, g, m);
    case 1: return tile_pair<R, RB, 1, REV, RC>(p, q, g, m);
    case 2: return tile_pair<R, RB, 2, REV, RC>(p, q, g, m);
    default: return tile_pair<R, RB, 3, REV, RC>(p, q, g, m);
  }
}

template <typename R, int RB, bool REV>
__device__ __forceinline__ R tile_gate(typename C2T<R>::T* p, typename C2T<R>::T* q, const TGate& g,
                                       const R* m, int gbase) {
  if ((gbase & g.cm_g) != g.cm_g) return 0;  // a group-bit control is 0 for this thread
  return g.cm_r ? tile_gate_rc<R, RB, REV, true>(p, q, g, m, gbase)
                : tile_gate_rc<R, RB, REV, false>(p, q, g, m, gbase);
}


// Forward (REV = false: psi only, gates in order) or reverse (REV = true:
// psi and lambda, gates in reverse order, gradient partials) over one block,
// for every tile of every parameter set of the chunk (gridDim.y = set).  One
// CTA per SM (the register arrays of both states need ~170 registers); the
// next tile streams into a second buffer with cp.async while the current one
// is processed.  Shared memory: two tile buffers (psi, then lambda in the
// reverse), the block's gate records and this set's matrices, then the
// per-warp gradient sums (reverse).
template <typename R, bool REV>
__global__ void __launch_bounds__(kTileThreads, 1)
    tile_sweep(typename C2T<R>::T* __restrict__ psi, typename C2T<R>::T* __restrict__ lam, uint64_t dim,
               TileGeom tg, const TGate* __restrict__ gates, int ngates, const TPhase* __restrict__ phases,
               int nph, const R* __restrict__ mats, uint64_t mat_stride, int ngrad, double* __restrict__ partial) {
  using T = typename C2T<R>::T;
  constexpr int TB = TileCfg<R>::TB, RB = TileCfg<R>::RB, NR = 1 << RB, TILE = 1 << TB;
  constexpr int BUF = (REV ? 2 : 1) * TILE;  // elements per buffer
  extern __shared__ __align__(16) unsigned char tsm[];
  T* bufs = reinterpret_cast<T*>(tsm);
  TGate* sg = reinterpret_cast<TGate*>(tsm + 2 * BUF * sizeof(T));
  R* smat = reinterpret_cast<R*>(sg + ngates);
  double* acc = reinterpret_cast<double*>(smat + 8 * (size_t)ngates);  // [warp][ngrad]
  __shared__ uint64_t off_lo[64], off_hi[64];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int set = blockIdx.y;
  T* s = psi + (uint64_t)set * dim;
  T* l = REV ? lam + (uint64_t)set * dim : nullptr;

  if (tid < 128) {
    const int half = tid >> 6, e = tid & 63;
    uint64_t off = 0;
    for (int b = 0; b < 6; ++b) {
      const int tb = 6 * half + b;
      if (tb < TB && ((e >> b) & 1)) off |= uint64_t{1} << tg.pos[tb];
    }
    (half ? off_hi : off_lo)[e] = off;
  }
  for (int i = tid; i < ngates; i += kTileThreads) {
    const TGate g = gates[i];
    sg[i] = g;
    const R* src = mats + ((uint64_t)g.mat * mat_stride + set) * 8;
#pragma unroll
    for (int k = 0; k < 8; ++k) smat[8 * i + k] = src[k];
  }
  if (REV)
    for (int i = tid; i < kTileWarps * ngrad; i += kTileThreads) acc[i] = 0.0;
  __syncthreads();

  auto tile_base = [&](uint64_t t) {
    uint64_t base = t;
#pragma unroll
    for (int b = 0; b < TB; ++b) {
      const int f = tg.pos[b];
      base = ((base >> f) << (f + 1)) | (base & ((uint64_t{1} << f) - 1));
    }
    return base;
  };
  auto prefetch = [&](uint64_t t, T* buf) {
    const uint64_t base = tile_base(t);
#pragma unroll 2
    for (int r = 0; r < NR; ++r) {
      const int e = tid + r * kTileThreads;
      const uint64_t o = base + (off_lo[e & 63] | off_hi[e >> 6]);
      tile_cp_async(buf + tphys<R>(e), s + o);
      if (REV) tile_cp_async(buf + TILE + tphys<R>(e), l + o);
    }
  };

  int cur = 0;
  if (blockIdx.x < tg.n_tiles) prefetch(blockIdx.x, bufs);
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  for (uint64_t t = blockIdx.x; t < tg.n_tiles; t += gridDim.x) {
    T* sp = bufs + cur * BUF;
    T* sl = sp + TILE;
    if (t + gridDim.x < tg.n_tiles) prefetch(t + gridDim.x, bufs + (cur ^ 1) * BUF);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // this tile's copies are done
    __syncthreads();
    for (int k = 0; k < nph; ++k) {
      const TPhase P = phases[REV ? nph - 1 - k : k];
      // group bits of this thread: the non-register tile bits, ascending
      int rmask = 0;
#pragma unroll
      for (int b = 0; b < RB; ++b) rmask |= 1 << P.r[b];
      int gbase = 0;
      {
        int kk = 0;
#pragma unroll
        for (int b = 0; b < TB; ++b)
          if (!((rmask >> b) & 1)) {
            gbase |= ((tid >> kk) & 1) << b;
            ++kk;
          }
      }
      // the swizzle is XOR-linear and gbase, rdep(j) have disjoint bits, so
      // the address of element j is tphys(gbase) ^ tphys(rdep(j))
      const int pg = tphys<R>(gbase);
      int pb[RB];
#pragma unroll
      for (int b = 0; b < RB; ++b) pb[b] = tphys<R>(1 << P.r[b]);
      T p[NR], q[NR];
#pragma unroll
      for (int j = 0; j < NR; ++j) {
        int a = pg;
#pragma unroll
        for (int b = 0; b < RB; ++b)
          if (j & (1 << b)) a ^= pb[b];
        p[j] = sp[a];
        if (REV) q[j] = sl[a];
      }
      for (int c = 0; c < P.count; ++c) {
        const int gi = REV ? P.first + P.count - 1 - c : P.first + c;
        const TGate g = sg[gi];
        const R part = tile_gate<R, RB, REV>(p, q, g, smat + 8 * gi, gbase);
        if (REV && g.grad >= 0) {
          double v = (double)part;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (lane == 0) acc[warp * ngrad + g.grad] += v;
        }
      }
      {
        // element addresses again, from a fresh read of the phase record (so
        // that the 2^RB addresses are not held in registers across the gates)
        unsigned rw;
        asm volatile("ld.global.nc.u32 %0, [%1];" : "=r"(rw) : "l"(&phases[REV ? nph - 1 - k : k]));
        const int pg2 = tphys<R>(gbase);
        int pb2[RB];
#pragma unroll
        for (int b = 0; b < RB; ++b) pb2[b] = tphys<R>(1 << ((rw >> (8 * b)) & 0xff));
#pragma unroll
        for (int j = 0; j < NR; ++j) {
          int a = pg2;
#pragma unroll
          for (int b = 0; b < RB; ++b)
            if (j & (1 << b)) a ^= pb2[b];
          sp[a] = p[j];
          if (REV) sl[a] = q[j];
        }
      }
      __syncthreads();
    }
    {
      const uint64_t base = tile_base(t);
      const volatile uint64_t* vlo = off_lo;
      const volatile uint64_t* vhi = off_hi;
#pragma unroll 2
      for (int r = 0; r < NR; ++r) {
        const int e = tid + r * kTileThreads;
        const uint64_t o = base + (vlo[e & 63] | vhi[e >> 6]);
        s[o] = sp[tphys<R>(e)];
        if (REV) l[o] = sl[tphys<R>(e)];
      }
    }
    __syncthreads();
    cur ^= 1;
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  if (REV)
    for (int g = tid; g < ngrad; g += kTileThreads) {
      double v = 0.0;
      for (int w = 0; w < kTileWarps; ++w) v += acc[w * ngrad + g];
      partial[((uint64_t)set * ngrad + g) * gridDim.x + blockIdx.x] = v;
    }
}


// The complex64 form of tile_sweep (same grid, pipeline and partials).
template <bool REV>
__global__ void __launch_bounds__(kTileThreads, 1)
    tile_sweep_c64(float2* __restrict__ psi, float2* __restrict__ lam, uint64_t dim, TileGeom tg,
                   const TGate* __restrict__ gates, int ngates, const TPhase* __restrict__ phases, int nph,
                   const float* __restrict__ mats, uint64_t mat_stride, int ngrad, double* __restrict__ partial) {
  constexpr int TB = TileCfg<float>::TB, RB = TileCfg<float>::RB, TILE = 1 << TB;
  static_assert(RB == 4, "8 packs of 2 amplitudes per state");
  constexpr int BUF = (REV ? 2 : 1) * TILE;
  extern __shared__ __align__(16) unsigned char tsm[];
  float2* bufs = reinterpret_cast<float2*>(tsm);
  f2* spk = reinterpret_cast<f2*>(tsm + 2 * BUF * sizeof(float2));  // [gate][16]
  TGate* sg = reinterpret_cast<TGate*>(spk + 16 * (size_t)ngates);
  double* acc = reinterpret_cast<double*>(sg + ngates);  // [warp][ngrad]
  __shared__ uint8_t sop[kMaxBlockGates];
  __shared__ uint64_t off_lo[64], off_hi[64];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int set = blockIdx.y;
  float2* s = psi + (uint64_t)set * dim;
  float2* l = REV ? lam + (uint64_t)set * dim : nullptr;

  if (tid < 128) {
    const int half = tid >> 6, e = tid & 63;
    uint64_t off = 0;
    for (int b = 0; b < 6; ++b) {
      const int tb = 6 * half + b;
      if (tb < TB && ((e >> b) & 1)) off |= uint64_t{1} << tg.pos[tb];
    }
    (half ? off_hi : off_lo)[e] = off;
  }
  for (int i = tid; i < ngates; i += kTileThreads) {
    const TGate g = gates[i];
    sg[i] = g;
    sop[i] = (uint8_t)pk_opcode(g, REV);
    const float* m = mats + ((uint64_t)g.mat * mat_stride + set) * 8;
    // U or U^dag, row-major (re, im) of entries 0..3
    float cr[4], ci[4];
    if (!REV) {
      for (int k = 0; k < 4; ++k) cr[k] = m[2 * k], ci[k] = m[2 * k + 1];
    } else {
      cr[0] = m[0], ci[0] = -m[1];
      cr[1] = m[4], ci[1] = -m[5];
      cr[2] = m[2], ci[2] = -m[3];
      cr[3] = m[6], ci[3] = -m[7];
    }
    f2* c = spk + 16 * i;
    for (int k = 0; k < 4; ++k) {
      c[2 * k] = pk2(cr[k], cr[k]);
      c[2 * k + 1] = pk2(ci[k], ci[k]);
      c[8 + k] = pk2(-ci[k], -ci[k]);
    }
    c[12] = pk2(cr[0], cr[3]);
    c[13] = pk2(ci[0], ci[3]);
    c[14] = pk2(-ci[0], -ci[3]);
    c[15] = 0;
  }
  if (REV)
    for (int i = tid; i < kTileWarps * ngrad; i += kTileThreads) acc[i] = 0.0;
  __syncthreads();

  auto tile_base = [&](uint64_t t) {
    uint64_t base = t;
#pragma unroll
    for (int b = 0; b < TB; ++b) {
      const int f = tg.pos[b];
      base = ((base >> f) << (f + 1)) | (base & ((uint64_t{1} << f) - 1));
    }
    return base;
  };
  auto prefetch = [&](uint64_t t, float2* buf) {
    const uint64_t base = tile_base(t);
#pragma unroll 2
    for (int r = 0; r < (1 << RB); ++r) {
      const int e = tid + r * kTileThreads;
      const uint64_t o = base + (off_lo[e & 63] | off_hi[e >> 6]);
      tile_cp_async(buf + tphys<float>(e), s + o);
      if (REV) tile_cp_async(buf + TILE + tphys<float>(e), l + o);
    }
  };

  int cur = 0;
  if (blockIdx.x < tg.n_tiles) prefetch(blockIdx.x, bufs);
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  for (uint64_t t = blockIdx.x; t < tg.n_tiles; t += gridDim.x) {
    float2* sp = bufs + cur * BUF;
    float2* sl = sp + TILE;
    if (t + gridDim.x < tg.n_tiles) prefetch(t + gridDim.x, bufs + (cur ^ 1) * BUF);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    __syncthreads();
    for (int k = 0; k < nph; ++k) {
      const TPhase P = phases[REV ? nph - 1 - k : k];
      int rmask = 0;
#pragma unroll
      for (int b = 0; b < RB; ++b) rmask |= 1 << P.r[b];
      int gbase = 0;
      {
        int kk = 0;
#pragma unroll
        for (int b = 0; b < TB; ++b)
          if (!((rmask >> b) & 1)) {
            gbase |= ((tid >> kk) & 1) << b;
            ++kk;
          }
      }
      const int pg = tphys<float>(gbase);
      int pb[RB];
#pragma unroll
      for (int b = 0; b < RB; ++b) pb[b] = tphys<float>(1 << P.r[b]);
      PackState A, L;
#pragma unroll
      for (int jo = 0; jo < 8; ++jo) {
        int a0 = pg;
#pragma unroll
        for (int b = 1; b < RB; ++b)
          if (jo & (1 << (b - 1))) a0 ^= pb[b];
        const int a1 = a0 ^ pb[0];
        const float2 x = sp[a0], y = sp[a1];
        A.r[jo] = pk2(x.x, y.x);
        A.i[jo] = pk2(x.y, y.y);
        if (REV) {
          const float2 u = sl[a0], v = sl[a1];
          L.r[jo] = pk2(u.x, v.x);
          L.i[jo] = pk2(u.y, v.y);
        }
      }
      for (int c = 0; c < P.count; ++c) {
        const int gi = REV ? P.first + P.count - 1 - c : P.first + c;
        const TGate g = sg[gi];
        float part = 0.f;
        if ((gbase & g.cm_g) == g.cm_g) part = pk_dispatch<REV>(sop[gi], A, L, g, spk + 16 * gi, gbase);
        if (REV && g.grad >= 0) {
          double v = (double)part;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (lane == 0) acc[warp * ngrad + g.grad] += v;
        }
      }
      {
        // addresses again from a fresh read of the phase record (not held
        // in registers across the gates)
        unsigned rw;
        asm volatile("ld.global.nc.u32 %0, [%1];" : "=r"(rw) : "l"(&phases[REV ? nph - 1 - k : k]));
        const int pg2 = tphys<float>(gbase);
        int pb2[RB];
#pragma unroll
        for (int b = 0; b < RB; ++b) pb2[b] = tphys<float>(1 << ((rw >> (8 * b)) & 0xff));
#pragma unroll
        for (int jo = 0; jo < 8; ++jo) {
          int a0 = pg2;
#pragma unroll
          for (int b = 1; b < RB; ++b)
            if (jo & (1 << (b - 1))) a0 ^= pb2[b];
          const int a1 = a0 ^ pb2[0];
          float xr, yr, xi, yi;
          upk2(A.r[jo], xr, yr);
          upk2(A.i[jo], xi, yi);
          sp[a0] = make_float2(xr, xi);
          sp[a1] = make_float2(yr, yi);
          if (REV) {
            upk2(L.r[jo], xr, yr);
            upk2(L.i[jo], xi, yi);
            sl[a0] = make_float2(xr, xi);
            sl[a1] = make_float2(yr, yi);
          }
        }
      }
      __syncthreads();
    }
    {
      const uint64_t base = tile_base(t);
      const volatile uint64_t* vlo = off_lo;
      const volatile uint64_t* vhi = off_hi;
#pragma unroll 2
      for (int r = 0; r < (1 << RB); ++r) {
        const int e = tid + r * kTileThreads;
        const uint64_t o = base + (vlo[e & 63] | vhi[e >> 6]);
        s[o] = sp[tphys<float>(e)];
        if (REV) l[o] = sl[tphys<float>(e)];
      }
    }
    __syncthreads();
    cur ^= 1;
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  if (REV)
    for (int g = tid; g < ngrad; g += kTileThreads) {
      double v = 0.0;
      for (int w = 0; w < kTileWarps; ++w) v += acc[w * ngrad + g];
      partial[((uint64_t)set * ngrad + g) * gridDim.x + blockIdx.x] = v;
    }
}

// Host plan of the tiled sweeps.
struct TBlock {
  TileGeom geom;
  int layer = 0;
  int gate_first = 0, n_gates = 0;    // into the concatenated TGate array
  int phase_first = 0, n_phases = 0;  // into the concatenated TPhase array
  std::vector<int> grad_gate;         // gradient slot -> gate list index
  size_t part_off = 0;                // into the gradient partials (doubles)
};

struct TilePlan {
  std::vector<TBlock> blocks;
  std::vector<TGate> gates;
  std::vector<TPhase> phases;
};

// Target tile bits, controls and kind of a lowered gate, in tile bits.
struct TileOp {
  uint8_t kind;
  int targets[2];
  int ntargets;
  int tgt_diag;  // kTDiag: target tile bit
  int cmask;     // controls (tile bits)
};

TileOp tile_op_of(const Pass& p, const int* tpos_of_qubit) {
  TileOp t{};
  auto tile_mask = [&](uint64_t m) {
    int r = 0;
    for (int q = 0; q < 64; ++q)
      if ((m >> q) & 1) r |= 1 << tpos_of_qubit[q];
    return r;
  };
  if (p.kind == PassKind::Phase) {
    // all fixed bits must be 1: the highest is the target, the rest controls
    const int top = p.fixed[p.nfixed - 1];
    t.kind = kTDiag;
    t.tgt_diag = tpos_of_qubit[top];
    t.cmask = tile_mask(p.p0 & ~(uint64_t{1} << top));
    t.ntargets = 0;
    return t;
  }
  const uint64_t diff = p.p0 ^ p.p1;
  if (p.mode == kPairDiag) {
    t.kind = kTDiag;
    t.tgt_diag = tpos_of_qubit[__builtin_ctzll(diff)];
    t.cmask = tile_mask(p.p0);
    t.ntargets = 0;
    return t;
  }
  if (__builtin_popcountll(diff) == 2) {
    t.kind = kTSwap2;
    const int a = __builtin_ctzll(diff), b = 63 - __builtin_clzll(diff);
    t.targets[0] = tpos_of_qubit[a];
    t.targets[1] = tpos_of_qubit[b];
    t.ntargets = 2;
    t.cmask = tile_mask(p.p0 & p.p1);
    return t;
  }
  t.kind = p.mode == kPairSwap ? kTPairSwap : kTPair;
  t.targets[0] = tpos_of_qubit[__builtin_ctzll(diff)];
  t.ntargets = 1;
  t.cmask = tile_mask(p.p0);
  return t;
}

template <typename R>
TilePlan plan_tiles(int n, const ketgpu_op* ops, const std::vector<int>& gate_ops, const std::vector<int>& layer_of,
                    const std::vector<GateGeom>& geo, const std::vector<uint8_t>& real, int seg_layers) {
  constexpr int TB = TileCfg<R>::TB, RB = TileCfg<R>::RB;
  constexpr bool kPacked = sizeof(R) == 4;  // complex64 sweeps pack pairs of amplitudes
  TilePlan tp;
  const int G = (int)gate_ops.size();
  std::vector<uint64_t> qmask(G);
  for (int i = 0; i < G; ++i) {
    const ketgpu_op& o = ops[gate_ops[i]];
    uint64_t m = 0;
    for (int j = 0; j < gate_arity(o.type); ++j) m |= uint64_t{1} << o.q[j];
    qmask[i] = m;
  }
  int i0 = 0;
  while (i0 < G) {
    // one checkpoint segment (seg_layers layers) at a time: blocks may run
    // across the layers of a segment but never across its ends
    int i1 = i0;
    while (i1 < G && layer_of[i1] / seg_layers == layer_of[i0] / seg_layers) ++i1;
    // A topological order of the layer that sweeps the qubits upwards: among
    // the gates whose predecessors (earlier gates sharing a qubit) are
    // placed, take the one with the lowest highest qubit.  Chains such as a
    // CX ring then fall into consecutive tiles instead of being cut by the
    // single-qubit gates listed before them.
    std::vector<int> rem;
    {
      std::vector<std::vector<int>> on_qubit(n);
      for (int i = i0; i < i1; ++i)
        for (int q = 0; q < n; ++q)
          if ((qmask[i] >> q) & 1) on_qubit[q].push_back(i);
      std::vector<size_t> head(n, 0);
      auto ready = [&](int i) {
        for (int q = 0; q < n; ++q)
          if (((qmask[i] >> q) & 1) && on_qubit[q][head[q]] != i) return false;
        return true;
      };
      using Key = std::pair<int, int>;  // (highest qubit, original index)
      std::priority_queue<Key, std::vector<Key>, std::greater<Key>> pq;
      std::vector<uint8_t> queued(G, 0);
      auto offer = [&](int i) {
        if (!queued[i] && ready(i)) {
          queued[i] = 1;
          pq.push({63 - __builtin_clzll(qmask[i]), i});
        }
      };
      for (int q = 0; q < n; ++q)
        if (!on_qubit[q].empty()) offer(on_qubit[q][0]);
      while (!pq.empty()) {
        const int i = pq.top().second;
        pq.pop();
        rem.push_back(i);
        for (int q = 0; q < n; ++q)
          if ((qmask[i] >> q) & 1) {
            ++head[q];
            if (head[q] < on_qubit[q].size()) offer(on_qubit[q][head[q]]);
          }
      }
    }
    while (!rem.empty()) {
      uint64_t S = 0x1f, blocked = 0;
      std::vector<int> take, keep;
      int ngrad = 0;
      for (int i : rem) {
        const bool grad = geo[i].gen && geo[i].pslot >= 0;
        const uint64_t u = S | qmask[i];
        if ((qmask[i] & blocked) || __builtin_popcountll(u) > TB || (int)take.size() >= kMaxBlockGates ||
            (grad && ngrad >= kMaxBlockGrads)) {
          blocked |= qmask[i];
          keep.push_back(i);
          continue;
        }
        S = u;
        take.push_back(i);
        ngrad += grad;
      }
      rem.swap(keep);
      for (int q = 0; q < n && __builtin_popcountll(S) < TB; ++q) S |= uint64_t{1} << q;
      TBlock b;
      b.layer = layer_of[i0];
      int tpos[64];
      for (int q = 0, k = 0; q < n; ++q)
        if ((S >> q) & 1) {
          b.geom.pos[k] = q;
          tpos[q] = k++;
        }
      for (int k = TB; k < 12; ++k) b.geom.pos[k] = 0;
      b.geom.n_tiles = uint64_t{1} << (n - TB);
      // phases: runs of gates whose target bits fit RB register bits
      std::vector<TileOp> top(take.size());
      for (size_t k = 0; k < take.size(); ++k) top[k] = tile_op_of(lower_gate(ops[gate_ops[take[k]]]), tpos);
      b.gate_first = (int)tp.gates.size();
      b.phase_first = (int)tp.phases.size();
      size_t k0 = 0;
      const int all_bits = (1 << TB) - 1;
      while (k0 < take.size()) {
        int rmask = 0;
        size_t k1 = k0;
        TPhase ph{};
        int slot_of[12];
        if (kPacked) {
          // complex64: register slot 0 is the pack bit, a tile bit that no
          // gate of the phase targets (pair kinds) or uses as a control;
          // the targets take at most the other RB - 1 slots
          int forbid = 0;
          for (; k1 < take.size(); ++k1) {
            int need = 0;
            for (int t = 0; t < top[k1].ntargets; ++t) need |= 1 << top[k1].targets[t];
            const int f = forbid | need | top[k1].cmask;
            if (__builtin_popcount(rmask | need) > RB - 1 || (f & all_bits) == all_bits) break;
            rmask |= need;
            forbid = f;
          }
          int pack = 0;
          while ((forbid >> pack) & 1) ++pack;
          for (int t = 0; t < TB && __builtin_popcount(rmask) < RB - 1; ++t)
            if (t != pack) rmask |= 1 << t;
          ph.r[0] = (uint8_t)pack;
          slot_of[pack] = 0;
          for (int t = 0, k = 1; t < TB; ++t)
            if ((rmask >> t) & 1) {
              ph.r[k] = (uint8_t)t;
              slot_of[t] = k++;
            }
          rmask |= 1 << pack;
        } else {
          for (; k1 < take.size(); ++k1) {
            int need = 0;
            for (int t = 0; t < top[k1].ntargets; ++t) need |= 1 << top[k1].targets[t];
            if (__builtin_popcount(rmask | need) > RB) break;
            rmask |= need;
          }
          for (int t = 0; t < TB && __builtin_popcount(rmask) < RB; ++t) rmask |= 1 << t;
          for (int t = 0, k = 0; t < TB; ++t)
            if ((rmask >> t) & 1) {
              ph.r[k] = (uint8_t)t;
              slot_of[t] = k++;
            }
        }
        ph.first = (int)tp.gates.size() - b.gate_first;  // relative to the block's first gate
        ph.count = (int)(k1 - k0);
        for (size_t k = k0; k < k1; ++k) {
          const TileOp& o = top[k];
          const int gi = take[k];
          TGate g{};
          g.kind = o.kind;
          g.mat = gi;
          g.gen = geo[gi].pslot >= 0 ? (uint8_t)geo[gi].gen : 0;
          g.real = real[gi];
          g.tslot = -1;
          int cm_r = 0, cm_g = 0;
          for (int t = 0; t < TB; ++t)
            if ((o.cmask >> t) & 1) {
              if ((rmask >> t) & 1) cm_r |= 1 << slot_of[t];
              else cm_g |= 1 << t;
            }
          g.cm_r = (uint8_t)cm_r;
          g.cm_g = (uint16_t)cm_g;
          if (o.kind == kTDiag) {
            g.tbit = (uint8_t)o.tgt_diag;
            if ((rmask >> o.tgt_diag) & 1) g.tslot = (int8_t)slot_of[o.tgt_diag];
          } else if (o.kind == kTSwap2) {
            const int a = slot_of[o.targets[0]], c = slot_of[o.targets[1]];
            g.s0 = (uint8_t)std::min(a, c);
            g.s1 = (uint8_t)std::max(a, c);
          } else {
            g.s0 = (uint8_t)slot_of[o.targets[0]];
          }
          g.grad = -1;
          if (g.gen) {
            g.grad = (int16_t)b.grad_gate.size();
            b.grad_gate.push_back(gi);
          }
          tp.gates.push_back(g);
        }
        tp.phases.push_back(ph);
        k0 = k1;
      }
      b.n_gates = (int)tp.gates.size() - b.gate_first;
      b.n_phases = (int)tp.phases.size() - b.phase_first;
      tp.blocks.push_back(std::move(b));
    }
    i0 = i1;
  }
  return tp;
}

// The tiled plan with blocks per layer, or per checkpoint segment of m
// layers when that needs fewer blocks (fewer HBM passes; a block that spans
// layers holds more gates and register phases, so on a tie the per-layer
// plan is kept).
template <typename R>
TilePlan plan_tiles_best(int n, const ketgpu_op* ops, const std::vector<int>& gate_ops,
                         const std::vector<int>& layer_of, const std::vector<GateGeom>& geo,
                         const std::vector<uint8_t>& real, int m) {
  TilePlan per_layer = plan_tiles<R>(n, ops, gate_ops, layer_of, geo, real, 1);
  if (m <= 1) return per_layer;
  TilePlan per_seg = plan_tiles<R>(n, ops, gate_ops, layer_of, geo, real, m);
  return per_seg.blocks.size() < per_layer.blocks.size() ? std::move(per_seg) : std::move(per_layer);
}

struct DevBuf {
  void* p = nullptr;
  explicit DevBuf(size_t b) { KB_CUDA(cudaMalloc(&p, b ? b : 8)); }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

int gen_of(int type) {
  switch (type) {
    case KETGPU_RX: case KETGPU_CRX: return 1;
    case KETGPU_RY: case KETGPU_CRY: return 2;
    case KETGPU_RZ: case KETGPU_CRZ: return 3;
    case KETGPU_CP: return 4;
    default: return 0;
  }
}

// ---------------------------------------------------------------------------
// Per-block complex64 kernels compiled at run time.  The compiled sweep
// (tile_sweep_c64) interprets each block's gate records: every gate goes
// through a switch, and the register moves at its merge points dominate the
// instruction count.  Here the block's phases and gates become compile-time
// constants of a kernel generated from adj_tile.cuh: a swap is a renaming,
// each gate is straight-line packed arithmetic.  The kernels are compiled
// with NVRTC for sm_100a (loaded with dlopen on first use), loaded with the
// runtime's library API and cached by their source text, so a layer
// structure that repeats is compiled once per process.  When NVRTC cannot
// be loaded or a compile fails, the compiled sweep runs instead.

const char* const kTileSource =
#include "adj_tile_src.inc"
    ;

struct Nvrtc {
  using Create = int (*)(void**, const char*, const char*, int, const char* const*, const char* const*);
  using Compile = int (*)(void*, int, const char* const*);
  using SizeOf = int (*)(void*, size_t*);
  using Get = int (*)(void*, char*);
  using Destroy = int (*)(void**);
  Create create = nullptr;
  Compile compile = nullptr;
  SizeOf log_size = nullptr, cubin_size = nullptr;
  Get log = nullptr, cubin = nullptr;
  Destroy destroy = nullptr;
  bool ok = false;
  Nvrtc() {
    const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
    void* h = nullptr;
    for (const char* n : names)
      if ((h = dlopen(n, RTLD_NOW | RTLD_LOCAL))) break;
    if (!h) return;
    create = reinterpret_cast<Create>(dlsym(h, "nvrtcCreateProgram"));
    compile = reinterpret_cast<Compile>(dlsym(h, "nvrtcCompileProgram"));
    log_size = reinterpret_cast<SizeOf>(dlsym(h, "nvrtcGetProgramLogSize"));
    log = reinterpret_cast<Get>(dlsym(h, "nvrtcGetProgramLog"));
    cubin_size = reinterpret_cast<SizeOf>(dlsym(h, "nvrtcGetCUBINSize"));
    cubin = reinterpret_cast<Get>(dlsym(h, "nvrtcGetCUBIN"));
    destroy = reinterpret_cast<Destroy>(dlsym(h, "nvrtcDestroyProgram"));
    ok = create && compile && log_size && log && cubin_size && cubin && destroy;
  }
};

Nvrtc& nvrtc() {
  static Nvrtc n;
  return n;
}

// AUTO uses the per-block kernels from this many qubits up.
constexpr int kJitMinQubits = 16;

std::mutex g_jit_mu;
std::map<std::string, cudaKernel_t> g_jit;  // source -> kernel (nullptr: failed)
std::string g_jit_last_log;

// Compile (once) and return the kernel "kb_tile_jit" of `src`, or nullptr.
cudaKernel_t jit_kernel(const std::string& src) {
  std::lock_guard<std::mutex> lock(g_jit_mu);
  auto it = g_jit.find(src);
  if (it != g_jit.end()) return it->second;
  cudaKernel_t k = nullptr;
  Nvrtc& nv = nvrtc();
  if (nv.ok) {
    const std::string full = std::string("#define KB_JIT 1\n") + kTileSource + src;
    void* prog = nullptr;
    if (nv.create(&prog, full.c_str(), "kb_tile_jit.cu", 0, nullptr, nullptr) == 0) {
      const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17"};
      const int rc = nv.compile(prog, 2, opts);
      size_t ls = 0;
      nv.log_size(prog, &ls);
      std::string lg(ls, '\0');
      if (ls) nv.log(prog, &lg[0]);
      g_jit_last_log = lg;
      size_t cs = 0;
      if (rc == 0 && nv.cubin_size(prog, &cs) == 0 && cs) {
        std::vector<char> cubin(cs);
        if (nv.cubin(prog, cubin.data()) == 0) {
          cudaLibrary_t lib = nullptr;
          if (cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) == cudaSuccess &&
              cudaLibraryGetKernel(&k, lib, "kb_tile_jit") != cudaSuccess)
            k = nullptr;
        }
      }
      nv.destroy(&prog);
    }
  }
  cudaGetLastError();  // a failed load leaves no sticky error behind
  g_jit[src] = k;
  return k;
}

int tphys_host(int e) { return e ^ (((e >> 4) ^ (e >> 8)) & 15); }

int pk_opcode_host(const TGate& g, bool rev) {
  const int rc = g.cm_r ? 1 : 0;
  const int gen = rev ? g.gen : 0;
  switch (g.kind) {
    case kTPair: return (g.s0 - 1) * 16 + (g.real ? 8 : 0) + gen * 2 + rc;
    case kTPairSwap: return 48 + (g.s0 - 1) * 2 + rc;
    case kTSwap2: return 54 + (g.s0 == 1 ? (g.s1 == 2 ? 0 : 1) : 2) * 2 + rc;
    default: return 60 + (g.tslot + 1) * 6 + (gen == 3 ? 1 : gen == 4 ? 2 : 0) * 2 + rc;
  }
}

// The kernel of one complex64 block: phases (in sweep order) and their gates
// as constants.  Parameters as tile_sweep_c64, without the phase table.
// Gradient slots per thread for a reverse block with `ngrad` gradients: the
// odd stride of the per-thread FP32 sums, or 0 for the per-tile warp
// reduction into per-warp FP64 sums (blocks with many gradients, whose
// per-thread slots would not leave room for two CTAs per SM).
constexpr int kThreadGradMax = 31;
int grad_slot_stride(int ngrad) { return ngrad > 0 && ngrad <= kThreadGradMax ? (ngrad | 1) : 0; }

std::string jit_source(const std::vector<TPhase>& phases, const std::vector<TGate>& gates, bool rev) {
  std::string o;
  auto line = [&](const std::string& x) { o += x + "\n"; };
  int ngrad_block = 0;
  for (const TGate& g : gates)
    if (g.grad >= 0) ngrad_block = std::max(ngrad_block, (int)g.grad + 1);
  const int gs = rev ? grad_slot_stride(ngrad_block) : 0;
  // Reverse: two CTAs per SM with one tile buffer each (load, compute,
  // store) beat one CTA with two buffers: the other CTA's work covers the
  // loads.  Forward: two CTAs, each prefetching its next tile.
  line("extern \"C\" __global__ void __launch_bounds__(256, 2)");
  line("kb_tile_jit(float2* psi, const float2* psi_src, float2* __restrict__ lam, uint64_t dim, kbt::TileGeom tg,");
  line("            const kbt::TGate* __restrict__ gates, int ngates, const float* __restrict__ mats,");
  line("            uint64_t mat_stride, int ngrad, double* __restrict__ partial) {");
  line("  using namespace kbt;");
  line(std::string("  constexpr bool REV = ") + (rev ? "true" : "false") + ";");
  line("  constexpr int TILE = 1 << TileCfg<float>::TB, BUF = (REV ? 2 : 1) * TILE;");
  line("  constexpr bool SINGLE = REV;  // one tile buffer");
  line("  extern __shared__ __align__(16) unsigned char tsm[];");
  line("  float2* bufs = reinterpret_cast<float2*>(tsm);");
  line("  f2* spk = reinterpret_cast<f2*>(tsm + (SINGLE ? 1 : 2) * BUF * sizeof(float2));");
  line("  float* accf = reinterpret_cast<float*>(spk + 16 * ngates);");
  line("  double* acc = reinterpret_cast<double*>(accf);");
  line("  constexpr int GS = " + std::to_string(gs) + ";  // per-thread gradient slots (0: per-warp sums)");
  line("  __shared__ uint64_t off_lo[64], off_hi[64];");
  line("  const int tid = threadIdx.x;");
  line("  const int set = blockIdx.y;");
  line("  float2* s = psi + (uint64_t)set * dim;  // tiles are stored here");
  line("  const float2* sin = psi_src + (uint64_t)set * dim;  // and loaded from here (psi, or a checkpoint)");
  line("  float2* l = REV ? lam + (uint64_t)set * dim : nullptr;");
  line("  c64_setup<REV>(tg, gates, ngates, mats, mat_stride, set, GS ? kTileThreads * GS : 2 * kTileWarps * ngrad,");
  line("                 off_lo, off_hi, spk, accf);");
  line("  __syncthreads();");
  line("  int cur = 0;");
  line("  if (!SINGLE && blockIdx.x < tg.n_tiles) c64_prefetch<REV>(tg, off_lo, off_hi, blockIdx.x, bufs, sin, l);");
  line("  asm volatile(\"cp.async.commit_group;\\n\" ::: \"memory\");");
  line("  for (uint64_t t = blockIdx.x; t < tg.n_tiles; t += gridDim.x) {");
  line("    float2* sp = bufs + (SINGLE ? 0 : cur) * BUF;");
  line("    float2* sl = sp + TILE;");
  line("    if (SINGLE) c64_prefetch<REV>(tg, off_lo, off_hi, t, bufs, sin, l);");
  line("    else if (t + gridDim.x < tg.n_tiles)");
  line("      c64_prefetch<REV>(tg, off_lo, off_hi, t + gridDim.x, bufs + (cur ^ 1) * BUF, sin, l);");
  line("    asm volatile(\"cp.async.commit_group;\\n\" ::: \"memory\");");
  line("    if (SINGLE) asm volatile(\"cp.async.wait_group 0;\\n\" ::: \"memory\");");
  line("    else asm volatile(\"cp.async.wait_group 1;\\n\" ::: \"memory\");");
  line("    __syncthreads();");
  constexpr int TB = TileCfg<float>::TB;
  const int nph = (int)phases.size();
  for (int k = 0; k < nph; ++k) {
    const TPhase& P = phases[rev ? nph - 1 - k : k];
    int rmask = 0;
    for (int b = 0; b < 4; ++b) rmask |= 1 << P.r[b];
    std::string gb = "0";
    for (int b = 0, kk = 0; b < TB; ++b)
      if (!((rmask >> b) & 1)) gb += " | (((tid >> " + std::to_string(kk++) + ") & 1) << " + std::to_string(b) + ")";
    line("    {");
    line("      const int gbase = " + gb + ";");
    line("      const int pg = tphys<float>(gbase);");
    line("      PackState A, L;");
    std::string pb;
    for (int b = 0; b < 4; ++b) pb += ", " + std::to_string(tphys_host(1 << P.r[b]));
    line("      c64_load_phase<REV>(sp, sl, pg" + pb + ", A, L);");
    for (int c = 0; c < P.count; ++c) {
      const int gi = rev ? P.first + P.count - 1 - c : P.first + c;
      const TGate& g = gates[gi];
      const int op = pk_opcode_host(g, rev);
      char buf[512];
      std::snprintf(buf, sizeof buf,
                    "      { constexpr TGate g{%d, %d, %d, %d, %d, %d, %d, %d, %d, %d, %d}; float part = 0.f;",
                    (int)g.kind, (int)g.s0, (int)g.s1, (int)g.tslot, (int)g.tbit, (int)g.cm_r, (int)(rev ? g.gen : 0),
                    (int)g.real, (int)g.cm_g, (int)g.grad, 0);  // mat: read from the gate table at set-up
      line(buf);
      const std::string call = "part = pk_exec<" + std::to_string(op) + ", REV>(A, L, g, spk + 16 * " +
                               std::to_string(gi) + ", gbase);";
      if (g.cm_g) line("        if ((gbase & " + std::to_string((int)g.cm_g) + ") == " + std::to_string((int)g.cm_g) +
                       ") " + call);
      else line("        " + call);
      if (rev && g.grad >= 0) {
        if (gs) line("        c64_grad_slot(accf, GS, " + std::to_string((int)g.grad) + ", part);");
        else line("        c64_grad(acc, ngrad, " + std::to_string((int)g.grad) + ", part);");
      }
      line("        (void)part; }");
    }
    line("      c64_store_phase<REV>(sp, sl, pg" + pb + ", A, L);");
    line("      __syncthreads();");
    line("    }");
  }
  line("    c64_store_tile<REV>(tg, off_lo, off_hi, t, sp, sl, s, l);");
  line("    __syncthreads();");
  line("    cur ^= 1;");
  line("  }");
  line("  asm volatile(\"cp.async.wait_all;\\n\" ::: \"memory\");");
  if (gs) line("  __syncthreads();");
  line(gs ? "  c64_flush_slots(accf, GS, ngrad, partial, set);" : "  if (REV) c64_flush(acc, ngrad, partial, set);");
  line("}");
  return o;
}

size_t jit_smem(bool rev, int ngates, int ngrad) {
  // forward: two buffers of psi; reverse: one buffer of psi and lambda, and
  // the gradient sums (per-thread FP32 slots or per-warp FP64)
  const int gs = grad_slot_stride(ngrad);
  const size_t acc = !rev ? 0 : gs ? (size_t)kTileThreads * gs * 4 : (size_t)kTileWarps * ngrad * 8;
  return 2 * (size_t{1} << TileCfg<float>::TB) * sizeof(float2) + (size_t)ngates * 16 * sizeof(f2) + acc;
}

// Dynamic shared memory of one tiled sweep launch (see the kernels).
template <typename R>
size_t tile_smem(bool rev, int ngates, int ngrad) {
  using T = typename C2T<R>::T;
  const size_t tiles = (rev ? 4 : 2) * (size_t{1} << TileCfg<R>::TB) * sizeof(T);
  const size_t per_gate = sizeof(R) == 4 ? 16 * sizeof(f2) + sizeof(TGate) : sizeof(TGate) + 8 * sizeof(R);
  return tiles + (size_t)ngates * per_gate + (rev ? (size_t)kTileWarps * ngrad * 8 : 0);
}

std::atomic<uint64_t> g_jit_launches{0};

template <typename R, bool REV>
void launch_tile(dim3 grid, cudaStream_t st, typename C2T<R>::T* psi, typename C2T<R>::T* lam, uint64_t dim,
                 const TBlock& b, const TGate* gates, const TPhase* phases, const R* mats, uint64_t chunk,
                 double* partial, cudaKernel_t jit = nullptr, const typename C2T<R>::T* psi_src = nullptr) {
  const int ngrad = REV ? (int)b.grad_gate.size() : 0;
  if constexpr (sizeof(R) == 4) {
    if (jit) {
      float2* a0 = psi;
      const float2* asrc = psi_src ? psi_src : psi;
      float2* a1 = lam;
      uint64_t d = dim;
      TileGeom tg = b.geom;
      const TGate* gp = gates + b.gate_first;
      int ng = b.n_gates;
      const float* mp = mats;
      uint64_t ms = chunk;
      int ngr = ngrad;
      double* pp = partial;
      void* args[] = {&a0, &asrc, &a1, &d, &tg, &gp, &ng, &mp, &ms, &ngr, &pp};
      KB_CUDA(cudaLaunchKernel(reinterpret_cast<const void*>(jit), grid, dim3(kTileThreads), args,
                               jit_smem(REV, b.n_gates, ngrad), st));
      count_launch();
      g_jit_launches.fetch_add(1, std::memory_order_relaxed);
      return;
    }
  }
  if (psi_src && psi_src != psi)  // the interpreted sweeps load in place only
    KB_CUDA(cudaMemcpyAsync(psi, psi_src, dim * sizeof(typename C2T<R>::T) * grid.y, cudaMemcpyDeviceToDevice, st));
  const size_t smem = tile_smem<R>(REV, b.n_gates, ngrad);
  if constexpr (sizeof(R) == 4)
    tile_sweep_c64<REV><<<grid, kTileThreads, smem, st>>>(psi, lam, dim, b.geom, gates + b.gate_first, b.n_gates,
                                                          phases + b.phase_first, b.n_phases, mats, chunk, ngrad,
                                                          partial);
  else
    tile_sweep<R, REV><<<grid, kTileThreads, smem, st>>>(psi, lam, dim, b.geom, gates + b.gate_first, b.n_gates,
                                                         phases + b.phase_first, b.n_phases, mats, chunk, ngrad,
                                                         partial);
  count_launch();
}

template <typename R>
void run_adjoint(int n, const ketgpu_op* ops, uint64_t nops, const int32_t* pidx, const double* params,
                 uint64_t nparams, uint64_t batch, const std::vector<uint64_t>& flip,
                 const std::vector<uint64_t>& sign, const std::vector<int>& phq, const double* coeffs,
                 int ckpt_every, int method, double* values, double* grads) {
  using T = typename C2T<R>::T;
  constexpr int TB = TileCfg<R>::TB;
  const uint64_t dim = uint64_t{1} << n;
  const int T_ = (int)flip.size();
  const bool tiled = method == KETGPU_ADJOINT_TILED || method == KETGPU_ADJOINT_TILED_JIT ||
                     (method == KETGPU_ADJOINT_AUTO && n >= TB);
  // per-block compiled kernels: complex64, asked for, or chosen at sizes
  // where the sweeps take long enough to repay a compile
  const bool want_jit = sizeof(R) == 4 && tiled &&
                        (method == KETGPU_ADJOINT_TILED_JIT || (method == KETGPU_ADJOINT_AUTO && n >= kJitMinQubits));
  if (tiled && n < TB)
    fail(KETGPU_ERR_INVALID, "adjoint: the tiled sweep needs at least " + std::to_string(TB) + " qubits");
  // gates (unitary ops) and layer boundaries (barriers)
  std::vector<int> gate_ops;
  std::vector<int> layer_of;
  int layer = 0;
  for (uint64_t i = 0; i < nops; ++i) {
    if (ops[i].type == KETGPU_BARRIER) {
      ++layer;
      continue;
    }
    if (!is_unitary(ops[i].type)) continue;
    gate_ops.push_back((int)i);
    layer_of.push_back(layer);
  }
  const int n_layers = layer + 1;
  const int m = ckpt_every > 0 ? ckpt_every : n_layers;
  const int n_ckpt = (n_layers + m - 1) / m;  // segment starts at layers 0, m, 2m, ...
  const size_t G = gate_ops.size();

  // memory: chunk of the batch that fits in ~60% of free memory
  size_t free_b = 0, total_b = 0;
  KB_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const size_t per_set = dim * sizeof(T) * (2 + (size_t)n_ckpt);
  if ((uint64_t)((free_b * 0.6) / per_set) < batch) {  // first take back ketgpu_run's kept state
    release_run_state();
    KB_CUDA(cudaMemGetInfo(&free_b, &total_b));
  }
  uint64_t chunk = std::max<uint64_t>(1, (uint64_t)((free_b * 0.6) / per_set));
  chunk = std::min<uint64_t>(chunk, batch);
  chunk = std::min<uint64_t>(chunk, 65535);

  cudaStream_t st;
  KB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{st};

  DevBuf psi(dim * sizeof(T) * chunk), lam(dim * sizeof(T) * chunk);
  DevBuf ck(dim * sizeof(T) * chunk * (size_t)n_ckpt);
  const int blocks = (int)std::min<uint64_t>(std::max<uint64_t>(1, (dim / 2 + kAThreads - 1) / kAThreads), 592);
  DevBuf mats(sizeof(double) * 8 * chunk * std::max<size_t>(G, 1));
  DevBuf hmeta(sizeof(uint64_t) * 2 * T_ + sizeof(int) * T_ + sizeof(double) * T_ + 64);
  {
    std::vector<char> h(sizeof(uint64_t) * 2 * T_ + sizeof(int) * T_ + sizeof(double) * T_);
    std::memcpy(h.data(), flip.data(), 8 * T_);
    std::memcpy(h.data() + 8 * T_, sign.data(), 8 * T_);
    std::memcpy(h.data() + 16 * T_, phq.data(), 4 * T_);
    std::memcpy(h.data() + 20 * T_, coeffs, 8 * T_);
    KB_CUDA(cudaMemcpyAsync(hmeta.p, h.data(), h.size(), cudaMemcpyHostToDevice, st));
  }
  // the terms with i^q folded into the coefficient, grouped by the top
  // qubit of their flip (ham_half; 0: same half, 1: other half)
  std::unique_ptr<DevBuf> d_ham;
  int ham_group0 = 0;
  const bool ham_split = T_ <= kHamSmemTerms && n >= 1;
  if (ham_split) {
    std::vector<HamTerm> ht;
    for (int pass = 0; pass < 2; ++pass)
      for (int t = 0; t < T_; ++t) {
        if ((int)((flip[t] >> (n - 1)) & 1) != pass) continue;
        HamTerm x;
        const double c = coeffs[t];
        x.flip = flip[t];
        x.sign = sign[t];
        switch (phq[t] & 3) {  // i^q
          case 0: x.cr = c, x.ci = 0.0; break;
          case 1: x.cr = 0.0, x.ci = c; break;
          case 2: x.cr = -c, x.ci = 0.0; break;
          default: x.cr = 0.0, x.ci = -c; break;
        }
        ht.push_back(x);
        if (pass == 0) ++ham_group0;
      }
    d_ham = std::make_unique<DevBuf>(sizeof(HamTerm) * std::max(T_, 1));
    KB_CUDA(cudaMemcpyAsync(d_ham->p, ht.data(), sizeof(HamTerm) * T_, cudaMemcpyHostToDevice, st));
    static bool ham_attr[2] = {false, false};
    if (!ham_attr[sizeof(R) == 8]) {
      KB_CUDA(cudaFuncSetAttribute(ham_half<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(sizeof(HamTerm) * kHamSmemTerms)));
      ham_attr[sizeof(R) == 8] = true;
    }
  }
  // ham_half grid: about one set's worth of resident CTAs per half
  const int ham_ctas = (int)std::min<uint64_t>(std::max<uint64_t>(1, (dim / 2 + kAThreads - 1) / kAThreads), 148ull * 8);
  const uint64_t* d_flip = hmeta.as<uint64_t>();
  const uint64_t* d_sign = d_flip + T_;
  const int* d_q = reinterpret_cast<const int*>(d_sign + T_);
  const double* d_coef = reinterpret_cast<const double*>(hmeta.as<char>() + 20 * T_);

  // geometry of every gate (independent of the parameters)
  std::vector<GateGeom> geo(G);
  for (size_t gi = 0; gi < G; ++gi) {
    const ketgpu_op& o = ops[gate_ops[gi]];
    const Pass p = lower_gate(o);
    GateGeom& g = geo[gi];
    g.nfixed = p.nfixed;
    for (int j = 0; j < 3; ++j) g.fixed[j] = p.fixed[j];
    g.count = dim >> p.nfixed;
    g.p0 = p.p0;
    g.p1 = p.p1;
    g.kind = p.kind == PassKind::Phase ? 2 : (p.mode == kPairSwap ? 1 : 0);
    const int32_t pi = pidx ? pidx[gate_ops[gi]] : -1;
    g.gen = pi >= 0 ? gen_of(o.type) : 0;
    g.pslot = pi;
    if (pi >= 0 && g.gen == 0) fail(KETGPU_ERR_INVALID, "adjoint: parameterised op must be Rx/Ry/Rz/CRx/CRy/CRz/CP");
    if (pi >= (int32_t)nparams) fail(KETGPU_ERR_OUT_OF_RANGE, "adjoint: parameter index out of range");
  }

  // per-set 2x2 of gate gi (U, row-major, FP64 interleaved).  The tiled
  // sweep stores a phase gate as diag(1, phase).
  auto gate_matrix = [&](size_t gi, uint64_t set, double* d) {
    ketgpu_op oo = ops[gate_ops[gi]];
    if (geo[gi].pslot >= 0) oo.p[0] = params[set * nparams + geo[gi].pslot];
    const Pass p = lower_gate(oo);
    cplx mm[4] = {p.m[0], p.m[1], p.m[2], p.m[3]};
    if (tiled && p.kind == PassKind::Phase) {
      mm[3] = p.m[0];
      mm[0] = cplx(1.0, 0.0);
      mm[1] = mm[2] = cplx(0.0, 0.0);
    }
    for (int j = 0; j < 4; ++j) {
      d[2 * j] = mm[j].real();
      d[2 * j + 1] = mm[j].imag();
    }
  };

  // tiled plan
  TilePlan tp;
  std::vector<cudaKernel_t> jit_fwd, jit_rev;
  std::unique_ptr<DevBuf> d_tgates, d_tphases;
  int gx = 1;
  size_t grad_doubles = 0;
  if (tiled) {
    std::vector<uint8_t> real(G, 1);
    double d[8];
    for (size_t gi = 0; gi < G; ++gi)
      for (uint64_t b = 0; b < batch && real[gi]; ++b) {
        gate_matrix(gi, b, d);
        if (d[1] != 0.0 || d[3] != 0.0 || d[5] != 0.0 || d[7] != 0.0) real[gi] = 0;
        if (geo[gi].pslot < 0) break;  // the same matrix for every set
      }
    tp = plan_tiles_best<R>(n, ops, gate_ops, layer_of, geo, real, m);
    d_tgates = std::make_unique<DevBuf>(sizeof(TGate) * std::max<size_t>(tp.gates.size(), 1));
    d_tphases = std::make_unique<DevBuf>(sizeof(TPhase) * std::max<size_t>(tp.phases.size(), 1));
    if (!tp.gates.empty())
      KB_CUDA(cudaMemcpyAsync(d_tgates->p, tp.gates.data(), sizeof(TGate) * tp.gates.size(),
                              cudaMemcpyHostToDevice, st));
    if (!tp.phases.empty())
      KB_CUDA(cudaMemcpyAsync(d_tphases->p, tp.phases.data(), sizeof(TPhase) * tp.phases.size(),
                              cudaMemcpyHostToDevice, st));
    if (want_jit && nvrtc().ok) {
      jit_fwd.assign(tp.blocks.size(), nullptr);
      jit_rev.assign(tp.blocks.size(), nullptr);
      for (size_t bi = 0; bi < tp.blocks.size(); ++bi) {
        const TBlock& b = tp.blocks[bi];
        const std::vector<TPhase> ph(tp.phases.begin() + b.phase_first,
                                     tp.phases.begin() + b.phase_first + b.n_phases);
        const std::vector<TGate> gs(tp.gates.begin() + b.gate_first, tp.gates.begin() + b.gate_first + b.n_gates);
        jit_fwd[bi] = jit_kernel(jit_source(ph, gs, false));
        jit_rev[bi] = jit_kernel(jit_source(ph, gs, true));
        if (jit_fwd[bi])
          KB_CUDA(cudaFuncSetAttribute(reinterpret_cast<const void*>(jit_fwd[bi]),
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)jit_smem(false, kMaxBlockGates, 0)));
        if (jit_rev[bi])
          KB_CUDA(cudaFuncSetAttribute(reinterpret_cast<const void*>(jit_rev[bi]),
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)std::max(jit_smem(true, kMaxBlockGates, kMaxBlockGrads),
                                                     jit_smem(true, kMaxBlockGates, kThreadGradMax))));
      }
    }
    const uint64_t n_tiles = uint64_t{1} << (n - TB);
    // About eight rounds of every resident CTA (two per SM) over the chunk's
    // sets, in whole rounds where the set count allows: a grid of 10 x 64
    // CTAs on 296 slots ran two full rounds and a third of 48 CTAs, leaving
    // most SMs idle for a third of each sweep.
    int sms = 148, dev = 0;
    KB_CUDA(cudaGetDevice(&dev));
    KB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const uint64_t slots = 2ull * (uint64_t)sms;
    gx = (int)std::min<uint64_t>(n_tiles, std::max<uint64_t>(1, (8 * slots + chunk / 2) / chunk));
    for (TBlock& b : tp.blocks) {
      b.part_off = grad_doubles;
      grad_doubles += b.grad_gate.size() * chunk * (size_t)gx;
    }
    static bool attr_set[2] = {false, false};
    if (!attr_set[sizeof(R) == 8]) {
      const int smem_rev = (int)tile_smem<R>(true, kMaxBlockGates, kMaxBlockGrads);
      const int smem_fwd = (int)tile_smem<R>(false, kMaxBlockGates, 0);
      if constexpr (sizeof(R) == 4) {
        KB_CUDA(cudaFuncSetAttribute(tile_sweep_c64<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_rev));
        KB_CUDA(cudaFuncSetAttribute(tile_sweep_c64<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_fwd));
      } else {
        KB_CUDA(cudaFuncSetAttribute(tile_sweep<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_rev));
        KB_CUDA(cudaFuncSetAttribute(tile_sweep<R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_fwd));
      }
      attr_set[sizeof(R) == 8] = true;
    }
  }
  const size_t ham_doubles = ham_split ? chunk * 2 * (size_t)ham_ctas : chunk * blocks;
  // gradient partials (tiled: per block; per-gate: [gate][set][block]), then
  // the expectation partials
  const size_t grad_region = tiled ? grad_doubles : (size_t)G * chunk * blocks;
  DevBuf part(sizeof(double) * (grad_region + ham_doubles));
  double* d_ham_part = part.as<double>() + grad_region;

  std::vector<double> hmats(8 * chunk * std::max<size_t>(G, 1));
  std::vector<R> hmats_t(tiled ? hmats.size() : 0);  // the tiled sweeps read them in the state's precision
  DevBuf mats_t(sizeof(R) * std::max<size_t>(hmats_t.size(), 1));
  std::vector<double> hpart;
  for (uint64_t b0 = 0; b0 < batch; b0 += chunk) {
    const uint64_t nb = std::min(chunk, batch - b0);
    for (size_t gi = 0; gi < G; ++gi)
      for (uint64_t b = 0; b < nb; ++b) gate_matrix(gi, b0 + b, &hmats[(gi * chunk + b) * 8]);
    KB_CUDA(cudaMemcpyAsync(mats.p, hmats.data(), sizeof(double) * 8 * chunk * std::max<size_t>(G, 1),
                            cudaMemcpyHostToDevice, st));
    if (tiled) {
      for (size_t i = 0; i < hmats.size(); ++i) hmats_t[i] = (R)hmats[i];
      KB_CUDA(cudaMemcpyAsync(mats_t.p, hmats_t.data(), sizeof(R) * hmats_t.size(), cudaMemcpyHostToDevice, st));
    }
    // With every block compiled, checkpoints cost no copies: the block
    // before a checkpoint writes its tiles into the checkpoint, the next
    // block reads them from there and writes psi (and in the reverse sweep
    // the first block of a segment reads psi from its checkpoint).
    bool ck_direct = tiled && !jit_fwd.empty();
    for (size_t bi = 0; ck_direct && bi < jit_fwd.size(); ++bi) ck_direct = jit_fwd[bi] && jit_rev[bi];
    auto ck_at = [&](int k) { return ck.as<T>() + (size_t)k * chunk * dim; };
    // forward
    T* ground = ck_direct ? ck_at(0) : psi.as<T>();
    KB_CUDA(cudaMemsetAsync(ground, 0, dim * sizeof(T) * nb, st));
    ground_batch<R><<<(unsigned)nb, 1, 0, st>>>(ground, dim);
    count_launch();
    // checkpoint k = the state at the start of layer k*m
    int next_ck = 0;
    auto store_ck = [&]() {
      KB_CUDA(cudaMemcpyAsync(ck.as<T>() + (size_t)next_ck * chunk * dim, psi.p, dim * sizeof(T) * nb,
                              cudaMemcpyDeviceToDevice, st));
      ++next_ck;
    };
    if (ck_direct) {
      const int B = (int)tp.blocks.size();
      const T* cur = ground;  // where the state lives now
      next_ck = 1;            // checkpoint 0 is the ground state
      for (int bi = 0; bi < B; ++bi) {
        const TBlock& b = tp.blocks[bi];
        if (cur != psi.as<T>() && next_ck < n_ckpt && next_ck * m <= b.layer) {
          // more checkpoints due here than blocks between them
          KB_CUDA(cudaMemcpyAsync(psi.p, cur, dim * sizeof(T) * nb, cudaMemcpyDeviceToDevice, st));
          cur = psi.as<T>();
        }
        while (cur == psi.as<T>() && next_ck < n_ckpt && next_ck * m <= b.layer) store_ck();
        T* out = psi.as<T>();
        if (bi + 1 < B && next_ck < n_ckpt && next_ck * m <= tp.blocks[bi + 1].layer) out = ck_at(next_ck++);
        dim3 grid((unsigned)gx, (unsigned)nb);
        launch_tile<R, false>(grid, st, out, nullptr, dim, b, d_tgates->as<TGate>(), d_tphases->as<TPhase>(),
                              mats_t.as<R>(), chunk, nullptr, jit_fwd[bi], cur);
        cur = out;
      }
      if (cur != psi.as<T>())
        KB_CUDA(cudaMemcpyAsync(psi.p, cur, dim * sizeof(T) * nb, cudaMemcpyDeviceToDevice, st));
    } else if (tiled) {
      for (const TBlock& b : tp.blocks) {
        while (next_ck < n_ckpt && next_ck * m <= b.layer) store_ck();
        dim3 grid((unsigned)gx, (unsigned)nb);
        launch_tile<R, false>(grid, st, psi.as<T>(), nullptr, dim, b, d_tgates->as<TGate>(), d_tphases->as<TPhase>(),
                              mats_t.as<R>(), chunk, nullptr,
                              jit_fwd.empty() ? nullptr : jit_fwd[&b - tp.blocks.data()]);
      }
    } else {
      for (size_t gi = 0; gi < G; ++gi) {
        while (next_ck < n_ckpt && next_ck * m <= layer_of[gi]) store_ck();
        dim3 grid((unsigned)blocks, (unsigned)nb);
        fwd_gate<R><<<grid, kAThreads, 0, st>>>(psi.as<T>(), dim, geo[gi], mats.as<double>() + gi * chunk * 8);
        count_launch();
      }
    }
    while (next_ck < n_ckpt) store_ck();
    KB_CUDA(cudaGetLastError());
    // lambda = H psi and <H>
    {
      if (ham_split) {
        KB_CUDA(cudaMemsetAsync(d_ham_part, 0, sizeof(double) * ham_doubles, st));
        const int g0 = ham_group0, g1 = T_ - ham_group0;
        dim3 hgrid((unsigned)ham_ctas, (unsigned)nb);
        for (int h = 0; h < 2; ++h) {
          if (g0 > 0) {
            ham_half<R><<<hgrid, kAThreads, sizeof(HamTerm) * g0, st>>>(
                psi.as<T>(), lam.as<T>(), dim, h, 1, g1 == 0 ? 1 : 0, d_ham->as<HamTerm>(), g0, d_ham_part);
            count_launch();
          }
          if (g1 > 0) {
            ham_half<R><<<hgrid, kAThreads, sizeof(HamTerm) * g1, st>>>(
                psi.as<T>(), lam.as<T>(), dim, h, g0 == 0 ? 1 : 0, 1, d_ham->as<HamTerm>() + g0, g1, d_ham_part);
            count_launch();
          }
        }
      } else {
        dim3 grid((unsigned)blocks, (unsigned)nb);
        ham_apply<R><<<grid, kAThreads, 0, st>>>(psi.as<T>(), lam.as<T>(), dim, d_flip, d_sign, d_q, d_coef, T_,
                                                 d_ham_part);
        count_launch();
      }
    }
    // reverse sweep; at the last gate (block) of each segment, walking
    // backwards, psi is reset to the checkpoint of the segment's end
    if (tiled) {
      const int B = (int)tp.blocks.size();
      for (int bi = B; bi-- > 0;) {
        const TBlock& b = tp.blocks[bi];
        const int seg = b.layer / m;
        const T* src = psi.as<T>();
        if (bi + 1 < B && tp.blocks[bi + 1].layer / m != seg && seg + 1 < n_ckpt) {
          if (ck_direct) src = ck_at(seg + 1);
          else
            KB_CUDA(cudaMemcpyAsync(psi.p, ck.as<T>() + (size_t)(seg + 1) * chunk * dim, dim * sizeof(T) * nb,
                                    cudaMemcpyDeviceToDevice, st));
        }
        dim3 grid((unsigned)gx, (unsigned)nb);
        launch_tile<R, true>(grid, st, psi.as<T>(), lam.as<T>(), dim, b, d_tgates->as<TGate>(),
                             d_tphases->as<TPhase>(), mats_t.as<R>(), chunk, part.as<double>() + b.part_off,
                             jit_rev.empty() ? nullptr : jit_rev[bi], src);
      }
    } else {
      for (size_t gi = G; gi-- > 0;) {
        const int seg = layer_of[gi] / m;
        if (gi + 1 < G && layer_of[gi + 1] / m != seg && seg + 1 < n_ckpt) {
          KB_CUDA(cudaMemcpyAsync(psi.p, ck.as<T>() + (size_t)(seg + 1) * chunk * dim, dim * sizeof(T) * nb,
                                  cudaMemcpyDeviceToDevice, st));
        }
        dim3 grid((unsigned)blocks, (unsigned)nb);
        rev_gate<R><<<grid, kAThreads, 0, st>>>(psi.as<T>(), lam.as<T>(), dim, geo[gi],
                                                mats.as<double>() + gi * chunk * 8,
                                                part.as<double>() + gi * chunk * blocks);
        count_launch();
      }
    }
    KB_CUDA(cudaGetLastError());
    const size_t part_count = grad_region + ham_doubles;
    hpart.resize(part_count);
    KB_CUDA(cudaMemcpyAsync(hpart.data(), part.p, sizeof(double) * part_count, cudaMemcpyDeviceToHost, st));
    KB_CUDA(cudaStreamSynchronize(st));
    const double* hham = hpart.data() + grad_region;
    for (uint64_t b = 0; b < nb; ++b) {
      double v = 0;
      const int per_set = ham_split ? 2 * ham_ctas : blocks;
      const double* pv = hham + b * per_set;
      for (int k = 0; k < per_set; ++k) v += pv[k];
      values[b0 + b] = v;
      double* gr = grads + (b0 + b) * nparams;
      for (uint64_t k = 0; k < nparams; ++k) gr[k] = 0.0;
      if (tiled) {
        for (const TBlock& blk : tp.blocks) {
          const size_t ng = blk.grad_gate.size();
          for (size_t k = 0; k < ng; ++k) {
            const size_t gi = (size_t)blk.grad_gate[k];
            const double* pg = &hpart[blk.part_off + (b * ng + k) * gx];
            double acc = 0;
            for (int c = 0; c < gx; ++c) acc += pg[c];
            gr[geo[gi].pslot] += (geo[gi].gen == 4) ? -2.0 * acc : acc;
          }
        }
      } else {
        for (size_t gi = 0; gi < G; ++gi) {
          if (geo[gi].pslot < 0) continue;
          double acc = 0;
          const double* pg = &hpart[gi * chunk * blocks + b * blocks];
          for (int k = 0; k < blocks; ++k) acc += pg[k];
          gr[geo[gi].pslot] += (geo[gi].gen == 4) ? -2.0 * acc : acc;
        }
      }
    }
  }
}

}  // namespace
}  // namespace kb

using namespace kb;

namespace {
int adjoint_entry(int32_t n, const ketgpu_op* ops, uint64_t n_ops, const int32_t* param_index, const double* params,
                  uint64_t n_params, uint64_t batch, const double* coeffs, const char* const* paulis,
                  uint64_t n_terms, int32_t precision, int32_t checkpoint_every, int32_t method, double* values,
                  double* grads) {
  try {
    if (n < 1 || n > 34) fail(KETGPU_ERR_INVALID, "adjoint: n_qubits must be in [1, 34]");
    if (!ops || !values || !grads || (n_params && !params) || !coeffs || !paulis || n_terms == 0)
      fail(KETGPU_ERR_INVALID, "adjoint: null argument");
    if (method < KETGPU_ADJOINT_AUTO || method > KETGPU_ADJOINT_TILED_JIT) fail(KETGPU_ERR_INVALID, "adjoint: bad method");
    validate_ops(n, ops, n_ops);
    std::vector<uint64_t> flip(n_terms), sign(n_terms);
    std::vector<int> q(n_terms);
    for (uint64_t t = 0; t < n_terms; ++t) pauli_masks(n, paulis[t], flip[t], sign[t], q[t]);
    if (precision == KETGPU_C64)
      run_adjoint<float>(n, ops, n_ops, param_index, params, n_params, batch, flip, sign, q, coeffs,
                         checkpoint_every, method, values, grads);
    else if (precision == KETGPU_C128)
      run_adjoint<double>(n, ops, n_ops, param_index, params, n_params, batch, flip, sign, q, coeffs,
                          checkpoint_every, method, values, grads);
    else
      fail(KETGPU_ERR_INVALID, "adjoint: bad precision");
    return KETGPU_OK;
  } catch (const Error& e) {
    kb::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    kb::set_last_error(e.what());
    return KETGPU_ERR_LOGIC;
  }
}
}  // namespace

KB_API int ketgpu_adjoint(int32_t n, const ketgpu_op* ops, uint64_t n_ops, const int32_t* param_index,
                          const double* params, uint64_t n_params, uint64_t batch, const double* coeffs,
                          const char* const* paulis, uint64_t n_terms, int32_t precision, int32_t checkpoint_every,
                          double* values, double* grads) {
  return adjoint_entry(n, ops, n_ops, param_index, params, n_params, batch, coeffs, paulis, n_terms, precision,
                       checkpoint_every, KETGPU_ADJOINT_AUTO, values, grads);
}

KB_API int ketgpu_adjoint_ex(int32_t n, const ketgpu_op* ops, uint64_t n_ops, const int32_t* param_index,
                             const double* params, uint64_t n_params, uint64_t batch, const double* coeffs,
                             const char* const* paulis, uint64_t n_terms, int32_t precision,
                             int32_t checkpoint_every, int32_t method, double* values, double* grads) {
  return adjoint_entry(n, ops, n_ops, param_index, params, n_params, batch, coeffs, paulis, n_terms, precision,
                       checkpoint_every, method, values, grads);
}

// Plan of the tiled sweeps as flat int32 records, for inspection and for
// checking the plan on the host: [n_blocks] then per block
// [layer, pos[12], n_phases, n_gates, phases (r0 r1 r2 r3 first count) ...,
//  gates (kind s0 s1 tslot tbit cm_r cm_g gen real grad op_index) ...],
// phase.first relative to the block's first gate.  Angles are taken from
// the ops as given (the real flag is per those angles).
KB_API int ketgpu_adjoint_plan_describe(int32_t n, const ketgpu_op* ops, uint64_t n_ops,
                                        const int32_t* param_index, int32_t precision, int32_t checkpoint_every,
                                        int32_t* out, uint64_t capacity, uint64_t* length) {
  try {
    if (!ops || !length) fail(KETGPU_ERR_INVALID, "adjoint_plan_describe: null argument");
    validate_ops(n, ops, n_ops);
    const int TB = precision == KETGPU_C64 ? TileCfg<float>::TB : TileCfg<double>::TB;
    if (n < TB) fail(KETGPU_ERR_INVALID, "adjoint_plan_describe: fewer qubits than a tile");
    std::vector<int> gate_ops, layer_of;
    int layer = 0;
    for (uint64_t i = 0; i < n_ops; ++i) {
      if (ops[i].type == KETGPU_BARRIER) {
        ++layer;
        continue;
      }
      if (!is_unitary(ops[i].type)) continue;
      gate_ops.push_back((int)i);
      layer_of.push_back(layer);
    }
    std::vector<GateGeom> geo(gate_ops.size());
    std::vector<uint8_t> real(gate_ops.size(), 0);
    for (size_t gi = 0; gi < gate_ops.size(); ++gi) {
      const ketgpu_op& o = ops[gate_ops[gi]];
      const int32_t pi = param_index ? param_index[gate_ops[gi]] : -1;
      geo[gi].pslot = pi;
      geo[gi].gen = pi >= 0 ? gen_of(o.type) : 0;
      const Pass p = lower_gate(o);
      bool r = true;
      for (int j = 0; j < 4; ++j) r = r && p.m[j].imag() == 0.0;
      real[gi] = r && p.kind == PassKind::Pair;
    }
    const int m = checkpoint_every > 0 ? checkpoint_every : layer + 1;
    const TilePlan tp = precision == KETGPU_C64 ? plan_tiles_best<float>(n, ops, gate_ops, layer_of, geo, real, m)
                                                : plan_tiles_best<double>(n, ops, gate_ops, layer_of, geo, real, m);
    std::vector<int32_t> v;
    v.push_back((int32_t)tp.blocks.size());
    for (const TBlock& b : tp.blocks) {
      v.push_back(b.layer);
      for (int k = 0; k < 12; ++k) v.push_back(b.geom.pos[k]);
      v.push_back(b.n_phases);
      v.push_back(b.n_gates);
      for (int k = 0; k < b.n_phases; ++k) {
        const TPhase& ph = tp.phases[b.phase_first + k];
        for (int j = 0; j < 4; ++j) v.push_back(ph.r[j]);
        v.push_back(ph.first);
        v.push_back(ph.count);
      }
      for (int k = 0; k < b.n_gates; ++k) {
        const TGate& g = tp.gates[b.gate_first + k];
        v.insert(v.end(), {g.kind, g.s0, g.s1, g.tslot, g.tbit, g.cm_r, g.cm_g, g.gen, g.real, g.grad,
                           gate_ops[g.mat]});
      }
    }
    *length = v.size();
    if (out) {
      if (capacity < v.size()) fail(KETGPU_ERR_INVALID, "adjoint_plan_describe: buffer too small");
      std::memcpy(out, v.data(), v.size() * sizeof(int32_t));
    }
    return KETGPU_OK;
  } catch (const Error& e) {
    kb::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    kb::set_last_error(e.what());
    return KETGPU_ERR_LOGIC;
  }
}

// Per-block compiled adjoint kernels: whether NVRTC could be loaded, how
// many distinct kernels are cached and how many launches used one.
KB_API int ketgpu_adjoint_jit_info(int32_t* available, uint64_t* kernels, uint64_t* launches) {
  try {
    if (available) *available = nvrtc().ok ? 1 : 0;
    if (kernels) {
      std::lock_guard<std::mutex> lock(g_jit_mu);
      uint64_t c = 0;
      for (const auto& kv : g_jit) c += kv.second != nullptr;
      *kernels = c;
    }
    if (launches) *launches = g_jit_launches.load();
    return KETGPU_OK;
  } catch (const std::exception& e) {
    kb::set_last_error(e.what());
    return KETGPU_ERR_LOGIC;
  }
}
