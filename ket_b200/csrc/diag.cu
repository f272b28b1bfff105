// diag.cu -- one pass for a run of diagonal gates.
//
// ket applies every diagonal gate as its own sweep: apply_cphase for CZ/CP
// (src/simulator.cpp:246-254, 323-324) and the single-qubit phases Z, S, T,
// Rz (:38-97) through apply_single.  Diagonal gates commute with each other,
// so a run of them (the planner collects every diagonal gate that can be moved
// to the front of what is left) is one diagonal operator.  Every gate of ket's
// set that is diagonal multiplies amplitude x by exp(i phi(x)) with phi linear
// in the index bits, or, for the two-qubit ones, bilinear in a pair of bits.
// So the run is
//   phi(x) = c0 + sum_i a_i x_i + sum_{i<j} b_ij x_i x_j.
//
// The kernel splits x into L = min(n, 12) low bits and n - L high bits.  The
// pair terms inside the low bits are one table of 2^L phases, built on the
// host in FP64.  A CTA handles 2^L consecutive amplitudes, whose high bits h
// are fixed.  For that chunk, the linear coefficients of the low bits
// (a_i + sum_j b_ij h_j) and the constant phi(h) fold into two 64-entry tables,
// built in FP64 with sincos.  Each amplitude then costs three complex products
// and one read and one write.  All phases are formed in FP64 and rounded to
// the state's precision for the products.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"

namespace kb {

bool is_diagonal_gate(int type) {
  switch (type) {
    case KETGPU_Z: case KETGPU_S: case KETGPU_SDG: case KETGPU_T: case KETGPU_TDG: case KETGPU_RZ:
    case KETGPU_CZ: case KETGPU_CP: case KETGPU_CRZ:
      return true;
    default:
      return false;
  }
}

// Phase terms of ket's diagonal gates (matrices as in single_matrix and
// lower_gate): Z diag(1,-1), S diag(1,i), Sdg diag(1,-i), T diag(1,e^{i pi/4}),
// Tdg its conjugate, Rz(t) diag(e^{-it/2}, e^{it/2}), CZ -1 on |11>, CP(l)
// e^{il} on |11>, CRz(t) Rz(t) on the target where the control is 1.
void add_diagonal_gate(const ketgpu_op& op, DiagPoly& poly, int n) {
  const double pi = 3.14159265358979323846;
  auto pair = [&](int i, int j, double v) {
    if (i > j) std::swap(i, j);
    poly.b[(size_t)i * n + j] += v;
  };
  const int q0 = op.q[0];
  switch (op.type) {
    case KETGPU_Z: poly.a[q0] += pi; break;
    case KETGPU_S: poly.a[q0] += pi / 2; break;
    case KETGPU_SDG: poly.a[q0] -= pi / 2; break;
    case KETGPU_T: poly.a[q0] += pi / 4; break;
    case KETGPU_TDG: poly.a[q0] -= pi / 4; break;
    case KETGPU_RZ:
      poly.c0 -= op.p[0] / 2;
      poly.a[q0] += op.p[0];
      break;
    case KETGPU_CZ: pair(op.q[0], op.q[1], pi); break;
    case KETGPU_CP: pair(op.q[0], op.q[1], op.p[0]); break;
    case KETGPU_CRZ:
      poly.a[op.q[0]] -= op.p[0] / 2;
      pair(op.q[0], op.q[1], op.p[0]);
      break;
    default:
      fail(KETGPU_ERR_LOGIC, "add_diagonal_gate: not a diagonal gate");
  }
}

// Device layout: table[2^L] (state precision, re/im), then FP64
// [c0, a[n], blh[L][H], bhh[H][H]] with H = n - L, blh[i][j] = b(i, L+j),
// bhh[j][k] = b(L+j, L+k) for j < k.
void diag_device_data(const DiagPoly& poly, int n, int precision, std::vector<unsigned char>& out) {
  const int L = std::min(n, kDiagLowBits), H = n - L;
  const size_t CH = size_t{1} << L;
  std::vector<double> q(CH, 0.0);
  for (size_t x = 1; x < CH; ++x) {
    const int top = 63 - __builtin_clzll(x);
    double v = q[x ^ (size_t{1} << top)];
    for (int i = 0; i < top; ++i)
      if ((x >> i) & 1) v += poly.b[(size_t)i * n + top];
    q[x] = v;
  }
  const size_t amp = precision == KETGPU_C64 ? 8 : 16;
  std::vector<double> prm;
  prm.push_back(poly.c0);
  for (int i = 0; i < n; ++i) prm.push_back(poly.a[i]);
  for (int i = 0; i < L; ++i)
    for (int j = 0; j < H; ++j) prm.push_back(poly.b[(size_t)i * n + L + j]);
  for (int j = 0; j < H; ++j)
    for (int k = 0; k < H; ++k) prm.push_back(k > j ? poly.b[(size_t)(L + j) * n + L + k] : 0.0);
  out.assign(CH * amp + prm.size() * sizeof(double), 0);
  for (size_t x = 0; x < CH; ++x) {
    const double c = std::cos(q[x]), s = std::sin(q[x]);
    if (precision == KETGPU_C64) {
      const float v[2] = {(float)c, (float)s};
      std::memcpy(&out[x * amp], v, sizeof v);
    } else {
      const double v[2] = {c, s};
      std::memcpy(&out[x * amp], v, sizeof v);
    }
  }
  std::memcpy(&out[CH * amp], prm.data(), prm.size() * sizeof(double));
}

namespace {

template <typename R>
struct CD;
template <>
struct CD<float> {
  using T = float2;
};
template <>
struct CD<double> {
  using T = double2;
};

template <typename T>
__device__ __forceinline__ T cmul(T a, T b) {
  T r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}

constexpr int kDiagThreads = 256;

template <typename R>
__global__ void __launch_bounds__(kDiagThreads)
    diag_kernel(typename CD<R>::T* __restrict__ s, int n, const typename CD<R>::T* __restrict__ table,
                const double* __restrict__ prm, uint64_t n_chunks) {
  using T = typename CD<R>::T;
  const int L = n < kDiagLowBits ? n : kDiagLowBits, H = n - L, CH = 1 << L;
  extern __shared__ __align__(16) unsigned char dsm[];
  T* q = reinterpret_cast<T*>(dsm);
  __shared__ T t1[64], t2[64];
  __shared__ double lin[kDiagLowBits];
  __shared__ double phih;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < CH; i += kDiagThreads) q[i] = table[i];
  const double c0 = prm[0];
  const double* a = prm + 1;
  const double* blh = a + n;
  const double* bhh = blh + L * H;
  for (uint64_t h = blockIdx.x; h < n_chunks; h += gridDim.x) {
    __syncthreads();  // the previous chunk's tables are no longer read
    if (warp == 0) {
      if (lane < L) {
        double v = a[lane];
        for (int j = 0; j < H; ++j)
          if ((h >> j) & 1) v += blh[lane * H + j];
        lin[lane] = v;
      }
    } else if (warp == 1) {
      double t = 0.0;
      if (lane < H && ((h >> lane) & 1)) {
        t = a[L + lane];
        for (int k = lane + 1; k < H; ++k)
          if ((h >> k) & 1) t += bhh[lane * H + k];
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      if (lane == 0) phih = c0 + t;
    }
    __syncthreads();
    if (tid < 64) {
      double ang = 0.0;
      for (int i = 0; i < (L < 6 ? L : 6); ++i)
        if ((tid >> i) & 1) ang += lin[i];
      double sn, cs;
      sincos(ang, &sn, &cs);
      t1[tid].x = (R)cs;
      t1[tid].y = (R)sn;
    } else if (tid < 128) {
      const int x = tid - 64;
      if (x < (1 << (L > 6 ? L - 6 : 0))) {
        double ang = phih;
        for (int i = 6; i < L; ++i)
          if ((x >> (i - 6)) & 1) ang += lin[i];
        double sn, cs;
        sincos(ang, &sn, &cs);
        t2[x].x = (R)cs;
        t2[x].y = (R)sn;
      }
    }
    __syncthreads();
    T* sb = s + (h << L);
    // all of the thread's amplitudes in flight before any arithmetic
    constexpr int kPer = (1 << kDiagLowBits) / kDiagThreads;
    T v[kPer];
#pragma unroll
    for (int r = 0; r < kPer; ++r) {
      const int e = tid + r * kDiagThreads;
      if (e < CH) v[r] = sb[e];
    }
#pragma unroll
    for (int r = 0; r < kPer; ++r) {
      const int e = tid + r * kDiagThreads;
      if (e < CH) sb[e] = cmul(v[r], cmul(cmul(t1[e & 63], t2[e >> 6]), q[e]));
    }
  }
}

}  // namespace

void launch_diag(const State& s, const Pass& p, const void* data) {
  (void)p;
  const int n = s.n;
  const int L = std::min(n, kDiagLowBits);
  const uint64_t n_chunks = uint64_t{1} << (n - L);
  const unsigned grid = (unsigned)std::min<uint64_t>(n_chunks, 148ull * 4);
  const size_t table = (size_t{1} << L) * s.amp_bytes();
  const double* prm = reinterpret_cast<const double*>(static_cast<const unsigned char*>(data) + table);
  if (s.precision == KETGPU_C64) {
    diag_kernel<float><<<grid, kDiagThreads, table, s.stream>>>(static_cast<float2*>(s.amps), n,
                                                               static_cast<const float2*>(data), prm, n_chunks);
  } else {
    static bool attr = false;
    if (!attr) {
      KB_CUDA(cudaFuncSetAttribute(diag_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)((size_t{1} << kDiagLowBits) * sizeof(double2))));
      attr = true;
    }
    diag_kernel<double><<<grid, kDiagThreads, table, s.stream>>>(static_cast<double2*>(s.amps), n,
                                                                static_cast<const double2*>(data), prm, n_chunks);
  }
  count_launch();
  KB_CUDA(cudaGetLastError());
}

}  // namespace kb
