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

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "internal.h"

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

template <typename R>
__global__ void ground_batch(typename C2T<R>::T* states, uint64_t dim) {
  typename C2T<R>::T one;
  one.x = 1;
  one.y = 0;
  states[(uint64_t)blockIdx.x * dim] = one;
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

template <typename R>
void run_adjoint(int n, const ketgpu_op* ops, uint64_t nops, const int32_t* pidx, const double* params,
                 uint64_t nparams, uint64_t batch, const std::vector<uint64_t>& flip,
                 const std::vector<uint64_t>& sign, const std::vector<int>& phq, const double* coeffs,
                 int ckpt_every, double* values, double* grads) {
  using T = typename C2T<R>::T;
  const uint64_t dim = uint64_t{1} << n;
  const int T_ = (int)flip.size();
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
  DevBuf part(sizeof(double) * chunk * blocks * (G + 1));
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

  std::vector<double> hmats(8 * chunk * std::max<size_t>(G, 1));
  std::vector<double> hpart;
  for (uint64_t b0 = 0; b0 < batch; b0 += chunk) {
    const uint64_t nb = std::min(chunk, batch - b0);
    // per-set matrices of every gate
    for (size_t gi = 0; gi < G; ++gi) {
      const ketgpu_op& o = ops[gate_ops[gi]];
      for (uint64_t b = 0; b < nb; ++b) {
        ketgpu_op oo = o;
        if (geo[gi].pslot >= 0) oo.p[0] = params[(b0 + b) * nparams + geo[gi].pslot];
        const Pass p = lower_gate(oo);
        double* d = &hmats[(gi * chunk + b) * 8];
        for (int j = 0; j < 4; ++j) {
          d[2 * j] = p.m[j].real();
          d[2 * j + 1] = p.m[j].imag();
        }
      }
    }
    KB_CUDA(cudaMemcpyAsync(mats.p, hmats.data(), sizeof(double) * 8 * chunk * std::max<size_t>(G, 1),
                            cudaMemcpyHostToDevice, st));
    // forward
    KB_CUDA(cudaMemsetAsync(psi.p, 0, dim * sizeof(T) * nb, st));
    ground_batch<R><<<(unsigned)nb, 1, 0, st>>>(psi.as<T>(), dim);
    count_launch();
    // checkpoint k = the state at the start of layer k*m
    int next_ck = 0;
    auto store_ck = [&]() {
      KB_CUDA(cudaMemcpyAsync(ck.as<T>() + (size_t)next_ck * chunk * dim, psi.p, dim * sizeof(T) * nb,
                              cudaMemcpyDeviceToDevice, st));
      ++next_ck;
    };
    for (size_t gi = 0; gi < G; ++gi) {
      while (next_ck < n_ckpt && next_ck * m <= layer_of[gi]) store_ck();
      dim3 grid((unsigned)blocks, (unsigned)nb);
      fwd_gate<R><<<grid, kAThreads, 0, st>>>(psi.as<T>(), dim, geo[gi], mats.as<double>() + gi * chunk * 8);
      count_launch();
    }
    while (next_ck < n_ckpt) store_ck();
    KB_CUDA(cudaGetLastError());
    // lambda = H psi and <H>
    {
      dim3 grid((unsigned)blocks, (unsigned)nb);
      ham_apply<R><<<grid, kAThreads, 0, st>>>(psi.as<T>(), lam.as<T>(), dim, d_flip, d_sign, d_q, d_coef, T_,
                                               part.as<double>() + (size_t)G * chunk * blocks);
      count_launch();
    }
    // reverse sweep; at the last gate of each segment (walking backwards)
    // psi is reset to the checkpoint of the segment's end
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
    KB_CUDA(cudaGetLastError());
    hpart.resize((G + 1) * chunk * blocks);
    KB_CUDA(cudaMemcpyAsync(hpart.data(), part.p, sizeof(double) * hpart.size(), cudaMemcpyDeviceToHost, st));
    KB_CUDA(cudaStreamSynchronize(st));
    for (uint64_t b = 0; b < nb; ++b) {
      double v = 0;
      const double* pv = &hpart[(size_t)G * chunk * blocks + b * blocks];
      for (int k = 0; k < blocks; ++k) v += pv[k];
      values[b0 + b] = v;
      double* gr = grads + (b0 + b) * nparams;
      for (uint64_t k = 0; k < nparams; ++k) gr[k] = 0.0;
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

}  // namespace
}  // namespace kb

using namespace kb;

KB_API int ketgpu_adjoint(int32_t n, const ketgpu_op* ops, uint64_t n_ops, const int32_t* param_index,
                          const double* params, uint64_t n_params, uint64_t batch, const double* coeffs,
                          const char* const* paulis, uint64_t n_terms, int32_t precision, int32_t checkpoint_every,
                          double* values, double* grads) {
  try {
    if (n < 1 || n > 34) fail(KETGPU_ERR_INVALID, "adjoint: n_qubits must be in [1, 34]");
    if (!ops || !values || !grads || (n_params && !params) || !coeffs || !paulis || n_terms == 0)
      fail(KETGPU_ERR_INVALID, "adjoint: null argument");
    validate_ops(n, ops, n_ops);
    std::vector<uint64_t> flip(n_terms), sign(n_terms);
    std::vector<int> q(n_terms);
    for (uint64_t t = 0; t < n_terms; ++t) pauli_masks(n, paulis[t], flip[t], sign[t], q[t]);
    if (precision == KETGPU_C64)
      run_adjoint<float>(n, ops, n_ops, param_index, params, n_params, batch, flip, sign, q, coeffs,
                         checkpoint_every, values, grads);
    else if (precision == KETGPU_C128)
      run_adjoint<double>(n, ops, n_ops, param_index, params, n_params, batch, flip, sign, q, coeffs,
                          checkpoint_every, values, grads);
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
