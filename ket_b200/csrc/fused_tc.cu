// fused_tc.cu -- dense k-qubit block apply on the 5th-generation tensor cores.
//
// The sm_100a replacement for ket's apply_matrix (src/simulator.cpp:357-393)
// when the fusion planner hands it a 2^k x 2^k complex block (k = 4 or 5) and
// the state is complex64.
//
// Formulation.  A tile is 128 groups x 2^k target combinations; group g's
// amplitudes, interleaved (re, im), form row g of A (K = 2^(k+1) floats).
// With B the real embedding of the block matrix M,
//     B[2c][2r] = Re M[r][c]   B[2c+1][2r] = -Im M[r][c]
//     B[2c][2r+1] = Im M[r][c] B[2c+1][2r+1] = Re M[r][c],
// the tile's output rows are D = A B, so the state is consumed in its own
// interleaved layout.  Precision: 3xTF32 -- A and B are split into
// hi = tf32(x) and lo = x - hi, and D = Ahi Bhi + Ahi Blo + Alo Bhi is
// accumulated in FP32 in tensor memory (tcgen05.mma kind::tf32, M=128,
// N=K=2^(k+1)).
//
// Pipeline (one CTA per SM, persistent over tiles, 256 threads):
//   cp.async (16 B, coalesced) raw tiles into a 3-slot ring -> all threads
//   split hi/lo into the 128B-swizzled K-major A images -> one thread issues
//   the MMAs, tcgen05.commit signals an mbarrier -> while tile j's MMAs run,
//   the CTA drains tile j-1's accumulator (double-buffered in TMEM) through
//   shared memory back to global memory in address order.  Two tiles of
//   loads stay in flight throughout.  Every mbarrier wait is bounded; on
//   timeout the kernel raises an error flag, drains its copies, frees its
//   tensor memory and returns.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "internal.h"

namespace kb {

__device__ int g_tc_error = 0;

namespace {

constexpr int kTcThreads = 256;
constexpr int kGroupBits = 7;  // M = 128 rows
constexpr int kSlots = 3;
constexpr uint32_t kWaitLimit = 1u << 26;

template <int KQ>
struct TcCfg {
  static constexpr int DIM = 1 << KQ;
  static constexpr int K = 2 * DIM;           // floats per A row
  static constexpr int N = 2 * DIM;           // accumulator columns
  static constexpr int TB = KQ + kGroupBits;  // tile bits
  static constexpr int TILE = 1 << TB;        // amplitudes per tile
  static constexpr int RAW_BYTES = TILE * 8;
  static constexpr int KBLK = (K * 4) / 128;      // 128-byte swizzle atoms along K
  static constexpr int A_BYTES = 128 * K * 4;     // one A image (hi or lo)
  static constexpr int B_BYTES = N * K * 4;       // one B image
  static constexpr int KSTEPS = K / 8;            // tf32 MMA K = 8
  static constexpr int TMEM_COLS = 2 * N;         // two accumulators
  static constexpr size_t SMEM = (size_t)kSlots * RAW_BYTES + 2 * A_BYTES + 2 * B_BYTES + 1024;
};

struct TcGeom {
  int tb;
  int tile_pos[16];
  int is_target[16];
  uint64_t n_tiles;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// K-major, 128-byte swizzle UMMA shared-memory descriptor (sm_100):
// start>>4 [0,14), LBO>>4 [16,30) (=1, unused for swizzled K-major),
// SBO>>4 [32,46) (=1024 B between 8-row groups), version 1 at bit 46,
// layout SWIZZLE_128B (2) at [61,64).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Byte offset of element (row, kk) of a K-major SW128 image with `rows` rows.
__host__ __device__ __forceinline__ uint32_t sw128_offset(int row, int kk, int rows) {
  const int kb = kk >> 5;             // 32 fp32 per 128-byte atom row
  const int chunk = (kk & 31) >> 2;   // 16-byte chunk in the row
  return (uint32_t)(kb * rows * 128 + row * 128 + ((chunk ^ (row & 7)) << 4) + ((kk & 3) << 2));
}

__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Bounded wait for the completion of the phase with the given parity.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (uint32_t it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                            uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

// 32 lanes x 16 columns (x16) of 32-bit accumulator per warp.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Instruction descriptor, kind::tf32: D=F32 [4,6), A=B=TF32 [7,10)/[10,13),
// both K-major, N>>3 at [17,23), M>>4 at [24,29).
template <int N>
__host__ __device__ constexpr uint32_t tf32_idesc() {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

template <int KQ>
__global__ void __launch_bounds__(kTcThreads, 1)
    fused_tc_kernel(float2* __restrict__ s, TcGeom g, const uint32_t* __restrict__ bimg) {
  using Cfg = TcCfg<KQ>;
  constexpr int DIM = Cfg::DIM, N = Cfg::N, TILE = Cfg::TILE;
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  // 1024-byte align the operand region for the 128B swizzle atoms.
  unsigned char* base_ptr =
      smem_dyn + ((1024 - (smem_u32(smem_dyn) & 1023)) & 1023);
  unsigned char* a_hi = base_ptr;
  unsigned char* a_lo = a_hi + Cfg::A_BYTES;
  unsigned char* b_hi = a_lo + Cfg::A_BYTES;
  unsigned char* b_lo = b_hi + Cfg::B_BYTES;
  unsigned char* raw = b_lo + Cfg::B_BYTES;  // kSlots x RAW_BYTES

  __shared__ uint64_t off_lo[64], off_hi[64];
  __shared__ int gc_lo[64], gc_hi[64];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base_slot;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // ---- lookup tables: address-order tile index e -> global offset / (g, c)
  if (tid < 128) {
    const int half = tid >> 6, e = tid & 63;
    uint64_t off = 0;
    int gc = 0, tcount = 0, gcount = 0;
    for (int j = 0; j < g.tb; ++j) {
      const bool t = g.is_target[j];
      const int sh = t ? tcount++ : (KQ + gcount++);
      const int local = j - 6 * half;
      if (local >= 0 && local < 6 && ((e >> local) & 1)) {
        off |= uint64_t{1} << g.tile_pos[j];
        gc |= 1 << sh;
      }
    }
    if (half == 0) {
      off_lo[e] = off;
      gc_lo[e] = gc;
    } else {
      off_hi[e] = off;
      gc_hi[e] = gc;
    }
  }
  // ---- B images (hi, lo) into shared memory
  {
    const uint4* src = reinterpret_cast<const uint4*>(bimg);
    uint4* dst = reinterpret_cast<uint4*>(b_hi);
    for (int i = tid; i < (2 * Cfg::B_BYTES) / 16; i += kTcThreads) dst[i] = src[i];
  }
  if (tid == 0) {
    mbar_init(smem_u32(&mbar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_slot)),
                 "n"(Cfg::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_proxy_async();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_slot;

  const uint64_t first = blockIdx.x;
  const uint64_t stride = gridDim.x;
  const uint64_t count = first < g.n_tiles ? (g.n_tiles - first + stride - 1) / stride : 0;

  auto tile_base = [&](uint64_t t) -> uint64_t {
    uint64_t b = t;
    for (int j = 0; j < g.tb; ++j) {
      const int f = g.tile_pos[j];
      b = ((b >> f) << (f + 1)) | (b & ((uint64_t{1} << f) - 1));
    }
    return b;
  };
  auto issue_load = [&](uint64_t j) {
    if (j < count) {
      const uint64_t base = tile_base(first + j * stride);
      const uint32_t slot = smem_u32(raw + (j % kSlots) * Cfg::RAW_BYTES);
      for (int ch = tid; ch < TILE / 2; ch += kTcThreads) {
        const int e = 2 * ch;
        const uint64_t off = off_lo[e & 63] + off_hi[e >> 6];
        cp_async16(slot + (uint32_t)e * 8u, s + base + off);
      }
    }
    cp_async_commit();
  };
  // Drain one accumulator through shared memory (slot `out`, [g][c ^ (g mod DIM)]).
  auto epilogue = [&](uint64_t j, unsigned char* out) {
    const int q = warp & 3, h = warp >> 2;
    const int row = 32 * q + lane;
    float2* o2 = reinterpret_cast<float2*>(out);
    const uint32_t acc = tmem + (uint32_t)((j & 1) * N);
#pragma unroll
    for (int part = 0; part < N / 2 / 16; ++part) {
      float v[16];
      tmem_ld16(acc + ((uint32_t)(32 * q) << 16) + (uint32_t)(h * (N / 2) + part * 16), v);
      tmem_ld_wait();
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int c = h * (DIM / 2) + part * 8 + i;
        o2[row * DIM + (c ^ (row & (DIM - 1)))] = make_float2(v[2 * i], v[2 * i + 1]);
      }
    }
    tc_fence_before();
    __syncthreads();
    const uint64_t base = tile_base(first + j * stride);
    for (int ch = tid; ch < TILE / 2; ch += kTcThreads) {
      const int e = 2 * ch;
      const int gc0 = gc_lo[e & 63] + gc_hi[e >> 6];
      const int gc1 = gc_lo[(e + 1) & 63] + gc_hi[(e + 1) >> 6];
      const int g0 = gc0 >> KQ, c0 = gc0 & (DIM - 1);
      const int g1 = gc1 >> KQ, c1 = gc1 & (DIM - 1);
      const float2 x = o2[g0 * DIM + (c0 ^ (g0 & (DIM - 1)))];
      const float2 y = o2[g1 * DIM + (c1 ^ (g1 & (DIM - 1)))];
      const uint64_t off = off_lo[e & 63] + off_hi[e >> 6];
      *reinterpret_cast<float4*>(s + base + off) = make_float4(x.x, x.y, y.x, y.y);
    }
    __syncthreads();
  };

  constexpr uint32_t idesc = tf32_idesc<N>();
  bool ok = true;

  issue_load(0);
  issue_load(1);
  issue_load(2);
  for (uint64_t j = 0; j < count && ok; ++j) {
    cp_async_wait<2>();
    __syncthreads();
    if (j >= 1) {
      const bool done = mbar_wait(smem_u32(&mbar), (uint32_t)((j - 1) & 1));
      if (__syncthreads_or(!done)) {  // the CTA leaves together
        ok = false;
        if (tid == 0) atomicExch(&g_tc_error, 1);
        break;
      }
      tc_fence_after();
    }
    // ---- split raw tile j into the swizzled hi/lo A images
    {
      const float4* r4 = reinterpret_cast<const float4*>(raw + (j % kSlots) * Cfg::RAW_BYTES);
      for (int ch = tid; ch < TILE / 2; ch += kTcThreads) {
        const float4 v = r4[ch];
        const int e = 2 * ch;
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int gc = gc_lo[(e + u) & 63] + gc_hi[(e + u) >> 6];
          const int row = gc >> KQ, c = gc & (DIM - 1);
          const float re = u ? v.z : v.x, im = u ? v.w : v.y;
          const float hr = tf32_hi(re), hi_ = tf32_hi(im);
          const uint32_t off = sw128_offset(row, 2 * c, 128);
          *reinterpret_cast<float2*>(a_hi + off) = make_float2(hr, hi_);
          *reinterpret_cast<float2*>(a_lo + off) = make_float2(re - hr, im - hi_);
        }
      }
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      const uint32_t acc = tmem + (uint32_t)((j & 1) * N);
      const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo);
      const uint32_t bh = smem_u32(b_hi), bl = smem_u32(b_lo);
#pragma unroll
      for (int st = 0; st < Cfg::KSTEPS; ++st) {
        const uint32_t ka = (uint32_t)((st >> 2) * 128 * 128 + (st & 3) * 32);
        const uint32_t kbo = (uint32_t)((st >> 2) * N * 128 + (st & 3) * 32);
        tc_mma_tf32(acc, sw128_desc(ah + ka), sw128_desc(bh + kbo), idesc, st > 0 ? 1u : 0u);
        tc_mma_tf32(acc, sw128_desc(ah + ka), sw128_desc(bl + kbo), idesc, 1u);
        tc_mma_tf32(acc, sw128_desc(al + ka), sw128_desc(bh + kbo), idesc, 1u);
      }
      tc_commit(smem_u32(&mbar));
    }
    if (j >= 1) epilogue(j - 1, raw + (j % kSlots) * Cfg::RAW_BYTES);
    else __syncthreads();
    issue_load(j + kSlots);
  }
  if (ok && count > 0) {
    const bool done = mbar_wait(smem_u32(&mbar), (uint32_t)((count - 1) & 1));
    if (__syncthreads_or(!done)) {
      ok = false;
      if (tid == 0) atomicExch(&g_tc_error, 1);
    } else {
      tc_fence_after();
      cp_async_wait<0>();
      __syncthreads();
      epilogue(count - 1, raw);
    }
  }
  cp_async_wait<0>();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(Cfg::TMEM_COLS)
                 : "memory");
  }
}

int sm_count_tc(int device) {
  int v = 0;
  KB_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device));
  return v;
}

template <int KQ>
void launch_tc(const State& st, const Pass& p, const void* b_image) {
  using Cfg = TcCfg<KQ>;
  TcGeom g{};
  g.tb = Cfg::TB;
  uint64_t tmask = 0;
  for (int b = 0; b < p.k; ++b) tmask |= uint64_t{1} << p.qubits[b];
  uint64_t tiles_mask = tmask;
  int extra = Cfg::TB - p.k;
  for (int q = 0; q < st.n && extra > 0; ++q)
    if (!((tmask >> q) & 1)) {
      tiles_mask |= uint64_t{1} << q;
      --extra;
    }
  if (extra > 0) fail(KETGPU_ERR_LOGIC, "tensor-core block needs n >= k + 7");
  int j = 0;
  for (int q = 0; q < st.n; ++q)
    if ((tiles_mask >> q) & 1) {
      g.tile_pos[j] = q;
      g.is_target[j] = (int)((tmask >> q) & 1);
      ++j;
    }
  g.n_tiles = st.dim() >> Cfg::TB;
  static int attr_done[64] = {0};
  if (st.device >= 0 && st.device < 64 && !(attr_done[st.device] & (1 << KQ))) {
    KB_CUDA(cudaFuncSetAttribute(fused_tc_kernel<KQ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)Cfg::SMEM));
    attr_done[st.device] |= 1 << KQ;
  }
  static int sms[64] = {0};
  if (!sms[st.device]) sms[st.device] = sm_count_tc(st.device);
  uint64_t grid = (uint64_t)sms[st.device];
  if (grid > g.n_tiles) grid = g.n_tiles;
  fused_tc_kernel<KQ><<<(unsigned)grid, kTcThreads, Cfg::SMEM, st.stream>>>(
      static_cast<float2*>(st.amps), g, static_cast<const uint32_t*>(b_image));
  count_launch();
  KB_CUDA(cudaGetLastError());
}

uint32_t host_tf32_rna(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return u & 0xffffe000u;  // inf / nan: truncate
  u += 0x1000u;  // round half away from zero on the magnitude
  return u & 0xffffe000u;
}

}  // namespace

bool tc_supported(int k) { return k == 4 || k == 5; }

size_t tc_image_bytes(int k) {
  const size_t dim = size_t{1} << k;
  return 2 * (2 * dim) * (2 * dim) * 4;
}

// B = real embedding of mat (row-major dim x dim complex), stored as the
// K-major SW128 images hi then lo (N rows of K floats each).
void build_tc_image(const std::vector<cplx>& mat, int k, std::vector<uint32_t>& out) {
  const int dim = 1 << k, K = 2 * dim, N = 2 * dim;
  out.assign(tc_image_bytes(k) / 4, 0u);
  unsigned char* hi = reinterpret_cast<unsigned char*>(out.data());
  unsigned char* lo = hi + (size_t)N * K * 4;
  for (int n = 0; n < N; ++n)
    for (int kk = 0; kk < K; ++kk) {
      const int r = n >> 1, c = kk >> 1;
      const cplx m = mat[(size_t)r * dim + c];
      double v;
      if ((n & 1) == 0) v = (kk & 1) == 0 ? m.real() : -m.imag();
      else v = (kk & 1) == 0 ? m.imag() : m.real();
      const float f = (float)v;
      const uint32_t h = host_tf32_rna(f);
      float hf;
      std::memcpy(&hf, &h, 4);
      const float l = f - hf;
      uint32_t lu;
      std::memcpy(&lu, &l, 4);
      const uint32_t off = sw128_offset(n, kk, N);
      std::memcpy(hi + off, &h, 4);
      std::memcpy(lo + off, &lu, 4);
    }
}

void launch_fused_tc(const State& s, const Pass& p, const void* b_image) {
  if (p.k == 5) launch_tc<5>(s, p, b_image);
  else if (p.k == 4) launch_tc<4>(s, p, b_image);
  else fail(KETGPU_ERR_LOGIC, "tensor-core block supports k = 4 or 5");
}

int tc_error_flag(bool reset) {
  int v = 0;
  KB_CUDA(cudaMemcpyFromSymbol(&v, g_tc_error, sizeof(int)));
  if (reset && v) {
    const int z = 0;
    KB_CUDA(cudaMemcpyToSymbol(g_tc_error, &z, sizeof(int)));
  }
  return v;
}

}  // namespace kb
