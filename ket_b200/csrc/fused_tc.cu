// fused_tc.cu -- dense k-qubit block apply on the 5th-generation tensor cores.
//
// The sm_100a replacement for ket's apply_matrix (src/simulator.cpp:357-393)
// when the fusion planner hands it a 2^k x 2^k complex block (k = 4, 5 or 6) and
// the state is complex64.
//
// Formulation.  A tile is 128 groups x 2^k target combinations; group g's
// amplitudes, interleaved (re, im), form row g of A (K = 2^(k+1) reals).
// With B the real embedding of the block matrix M,
//     B[2c][2r] = Re M[r][c]   B[2c+1][2r] = -Im M[r][c]
//     B[2c][2r+1] = Im M[r][c] B[2c+1][2r+1] = Re M[r][c],
// the tile's output rows are D = A B, so the state is consumed in its own
// interleaved layout.  Precision: 3xFP16 with power-of-two scaling.  Each A
// row is scaled by 2^s (its largest magnitude into [2^14, 2^15)) and B by
// 2^sb, both split into hi = fp16(x) and lo = fp16(x - hi) (11 significant
// bits each, the split of 3xTF32), and D = Ahi Bhi + Ahi Blo + Alo Bhi is
// accumulated in FP32 in tensor memory (tcgen05.mma kind::f16, M=128,
// N=K=2^(k+1)) and scaled back by 2^-(s+sb) in the epilogue.  The scaling
// keeps both halves in fp16's normal range whatever the amplitudes'
// magnitude, so an element's error stays within 2^-22 of itself plus
// 2^-39 of its row's largest; fp16 halves run the MMAs at twice the TF32
// rate and take half the tensor and shared memory.
//
// Pipeline (one CTA per SM, persistent over tiles, warp-specialised):
//   raw tiles into a ring of staging images -- one tiled tensor copy per
//   tile (two half-tile copies for k = 6) when qubits 0 and 1 are group
//   bits, per-thread cp.async otherwise -> converter warps scale and split
//   hi/lo into tensor memory (two A regions, tile parity) -> one thread
//   issues the MMAs, tcgen05.commit signals an mbarrier -> while tile j's
//   MMAs run, the epilogue drains tile j-1's accumulator (double-buffered in
//   TMEM) back to global memory, straight from registers or through shared
//   memory.  Every mbarrier wait is bounded; on timeout the kernel raises an
//   error flag, drains its copies, frees its tensor memory and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "internal.h"

namespace kb {

__device__ int g_tc_error = 0;

namespace {

constexpr int kTcThreads = 416;
constexpr int kGroupBits = 7;  // M = 128 rows
constexpr uint32_t kWaitLimit = 1u << 26;
constexpr int kSmemBudget = 232448 - 1024;  // opt-in limit less static shared memory

template <int KQ>
struct TcCfg {
  static constexpr int DIM = 1 << KQ;
  static constexpr int K = 2 * DIM;           // reals per A row
  static constexpr int N = 2 * DIM;           // accumulator columns
  static constexpr int TB = KQ + kGroupBits;  // tile bits
  static constexpr int TILE = 1 << TB;        // amplitudes per tile
  static constexpr int RAW_BYTES = TILE * 8;  // one staging image (the FP32 tile)
  // one fp16 B image: whole 128-byte swizzle atoms (64 halves) along K, so
  // k = 4 (K = 32) leaves the upper half of each atom row unused
  static constexpr int B_BYTES = (K + 63) / 64 * N * 128;
  static constexpr int KSTEPS = K / 16;       // f16 MMA K = 16
  // Tensor memory: two A regions (tile parity), each hi | lo with two fp16
  // per 32-bit column (K columns), and two accumulator regions of N FP32
  // columns; all three products of a tile go into one accumulator.
  static constexpr int A_COLS = K;
  static constexpr int TMEM_COLS = 2 * A_COLS + 2 * N;
  // staging images: as many as fit next to the B images (loads in flight)
  static constexpr int SLOTS_FIT = (kSmemBudget - 1024 - 2 * B_BYTES) / RAW_BYTES;
  static constexpr int SLOTS = SLOTS_FIT > 12 ? 12 : SLOTS_FIT;
  // k = 6 with a tensor copy: half-tile staging slots (the tile split by its
  // highest target qubit), so copies run further ahead of the converters
  static constexpr bool HALVES = KQ == 6;
  static constexpr int HALF_BYTES = RAW_BYTES / 2;
  static constexpr int HSLOTS = HALVES ? (kSmemBudget - 1024 - 2 * B_BYTES) / HALF_BYTES : 0;
  static constexpr int SB = SLOTS > HSLOTS ? SLOTS : HSLOTS;  // barrier pairs
  static constexpr size_t STAGE = (size_t)SLOTS * RAW_BYTES > (size_t)HSLOTS * HALF_BYTES
                                      ? (size_t)SLOTS * RAW_BYTES
                                      : (size_t)HSLOTS * HALF_BYTES;
  static constexpr size_t SMEM = STAGE + 2 * B_BYTES + 1024;  // + alignment slack
  static_assert(TMEM_COLS <= 512 && (TMEM_COLS & (TMEM_COLS - 1)) == 0, "tensor memory budget");
  static_assert(SLOTS >= (HALVES ? 2 : 3), "shared memory budget");
  static_assert(!HALVES || HSLOTS >= 4, "shared memory budget");
  static_assert(SMEM <= (size_t)kSmemBudget + 1024, "shared memory budget");
};

struct TcGeom {
  int tile_pos[16];   // tile qubits, ascending
  int is_target[16];
  int m_low;          // tile qubits 0..m_low-1 form the low run
  int nh;             // tile qubits above the low run
  int hpos[16];
  int direct;         // the epilogue stores from registers (see launch_fused_tc)
  // Tensor-copy producer (tma_dims > 0, see launch_tc): dimension i of the
  // tensor map starts at qubit tma_start[i]; a tile's coordinate in it is
  // (base >> tma_start[i]) & tma_mask[i].  ctile[c] = swizzled byte offset of
  // combination c in the tile image (natural tile index order).
  int tma_dims;
  int tma_start[5];
  uint64_t tma_mask[5];
  uint32_t ctile[64];
  uint64_t cdep[64];  // offset of target combination c from its group's amplitude
  uint64_t n_tiles;
  // k = 6 tensor copy in half tiles (half = 1): each tile is two boxes of
  // the tensor map over the tile less its highest target qubit, at the tile
  // base and at base + top_off; ctile[0..31] are the low five targets'
  // offsets in a half box and gbit_off[b] is group bit b's.
  int half;
  uint64_t top_off;
  uint32_t gbit_off[kGroupBits];
  // non-null: the epilogue also sums |out|^2 in FP64 and CTA b writes its sum
  // to norm_out[b]
  double* norm_out;
  // cp.async producers and staged stores: chunk i of thread t covers tile
  // amplitudes e = 2t + 256i and e + 1; its offsets are those of e = 2t
  // XOR those of e = 256i (amp_offsets is XOR-linear in e), and these tables
  // hold the latter: state offset, A-layout (input) and staging (output)
  // byte offsets
  uint64_t chunk_g[32];
  uint32_t chunk_s_in[32], chunk_s_out[32];
};

// Output staging when qubit 0 is a group bit: amplitudes e and e+1 (rows
// r and r+64, same combination c) side by side in one 16-byte slot, slot
// (r mod 64) * dim + (c ^ (r mod 8)), so the store phase reads one 16-byte
// word per chunk and the TMEM drain writes stay spread over the banks.
__host__ __device__ inline uint32_t pair_slot_offset(int row, int comb, int dim) {
  return (uint32_t)(((row & 63) * dim + (comb ^ (row & 7))) * 16 + 8 * (row >> 6));
}

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

// Byte offset of FP32 element (row, kk) of a K-major SW128 image with `rows`
// rows (the staging images).
__host__ __device__ __forceinline__ uint32_t sw128_offset(int row, int kk, int rows) {
  const int kb = kk >> 5;             // 32 fp32 per 128-byte atom row
  const int chunk = (kk & 31) >> 2;   // 16-byte chunk in the row
  return (uint32_t)(kb * rows * 128 + row * 128 + ((chunk ^ (row & 7)) << 4) + ((kk & 3) << 2));
}

// Byte offset of fp16 element (row, kk) of a K-major SW128 image with `rows`
// rows (the B images).
__host__ __device__ __forceinline__ uint32_t sw128_offset_h(int row, int kk, int rows) {
  const int kb = kk >> 6;             // 64 fp16 per 128-byte atom row
  const int chunk = (kk & 63) >> 3;   // 16-byte chunk in the row
  return (uint32_t)(kb * rows * 128 + row * 128 + ((chunk ^ (row & 7)) << 4) + ((kk & 7) << 1));
}

// Offsets of tile amplitude e (address order: bit j of e <-> qubit
// tile_pos[j]): from the tile base in the state (goff), and in bytes in an
// A-layout image (soff: row = group, with a group bit at qubit 0 rotated to
// row bit 6, kk = 2*comb), or with out_layout and qubit 0 a group bit in the
// paired output staging.  Both are XOR-linear in e: e's bits land on
// disjoint positions, and the swizzles XOR disjoint fields.
__host__ __device__ inline void amp_offsets(const TcGeom& g, int tb, int dim, int e, bool out_layout,
                                            uint64_t* goff, uint32_t* soff) {
  const bool q0_group = !g.is_target[0];
  uint64_t off = 0;
  int grp = 0, comb = 0, gb = 0, cb = 0;
  for (int j = 0; j < tb; ++j) {
    const int bit = (e >> j) & 1;
    if (g.is_target[j]) comb |= bit << cb++;
    else grp |= bit << gb++;
    if (bit) off |= uint64_t{1} << g.tile_pos[j];
  }
  const int row = q0_group ? ((grp >> 1) | ((grp & 1) << (kGroupBits - 1))) : grp;
  *goff = off;
  *soff = (out_layout && q0_group) ? pair_slot_offset(row, comb, dim) : sw128_offset(row, 2 * comb, 128);
}

// Packed FP32 pairs (sm_100 f32x2 instructions: two FP32 operations each).
using f32x2 = unsigned long long;
__device__ __forceinline__ f32x2 pack2(float lo, float hi) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ float2 unpack2(f32x2 v) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
  return r;
}
__device__ __forceinline__ f32x2 mul_x2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 fma_x2(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t saddr, const void* g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(saddr), "l"(g) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// One tiled tensor copy (2 to 5 dimensions, no multicast) of a whole box
// into shared memory, completing its bytes on the mbarrier at `bar`.
__device__ __forceinline__ void tma_load_box(uint32_t dst, const CUtensorMap* map, const int* c, int dims,
                                             uint32_t bar) {
  const uint64_t m = reinterpret_cast<uint64_t>(map);
  switch (dims) {
    case 2:
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
          "[%4];" ::"r"(dst),
          "l"(m), "r"(c[0]), "r"(c[1]), "r"(bar)
          : "memory");
      break;
    case 3:
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
          "%4}], [%5];" ::"r"(dst),
          "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(bar)
          : "memory");
      break;
    case 4:
      asm volatile(
          "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
          "%4, %5}], [%6];" ::"r"(dst),
          "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(bar)
          : "memory");
      break;
    default:
      asm volatile(
          "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
          "%4, %5, %6}], [%7];" ::"r"(dst),
          "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(bar)
          : "memory");
      break;
  }
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
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

// A from tensor memory (lanes = rows, two fp16 of K per 32-bit column), B
// from shared memory, D in tensor memory (FP32).
__device__ __forceinline__ void tc_mma_f16_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc,
                                              uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// 32 lanes x 16 columns of 32-bit values from the warp's registers.  No
// memory clobber: the store reads registers only, and as volatile asm it
// keeps its order against the tcgen05 waits and fences, so the compiler may
// move shared-memory reads of the next columns ahead of it.
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
          taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
      "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]));
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

// 32 lanes x NC columns of 32-bit accumulator per warp.
template <int NC>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float* v);
template <>
__device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, float* v) {
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

// Instruction descriptor, kind::f16: D=F32 [4,6), A=B=F16 (0) [7,10)/[10,13),
// both K-major, N>>3 at [17,23), M>>4 at [24,29).
template <int N>
__host__ __device__ constexpr uint32_t f16_idesc() {
  static_assert(N % 16 == 0 && N >= 16 && N <= 256, "M = 128 needs N a multiple of 16 in [16, 256]");
  return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// Roles (13 warps): 0-3 producers (cp.async into staging images; with a
// tensor map, thread 0 alone issues one tiled copy per tile or half tile),
// 4-7 converters (scale and hi/lo split into the A regions), 8-11 epilogue
// (TMEM -> HBM, from registers or through a staging image; warp w reads TMEM
// lanes 32*(w%4)..+31), 12 the MMA issuer.  mbarriers hand each tile from
// stage to stage, so loads of later tiles, the split of tile j+1, the MMAs of
// tile j and the drain of tile j-1 proceed concurrently.
constexpr int kProducers = 128, kConverters = 128, kEpilogue = 128;
constexpr int kScaleRing = 4;  // row scales in flight (see the converters)

// NORM: the epilogue also sums |out|^2 into g.norm_out (the plan's last
// block before its norm restore); a separate instantiation, so the common
// one carries none of it.
template <int KQ, bool NORM>
__global__ void __launch_bounds__(kTcThreads, 1)
    fused_tc_kernel(float2* __restrict__ s, TcGeom g, const uint32_t* __restrict__ bimg,
                    const __grid_constant__ CUtensorMap tmap) {
  using Cfg = TcCfg<KQ>;
  constexpr int N = Cfg::N, TILE = Cfg::TILE, DIM = Cfg::DIM;
  constexpr int CPT = TILE / 2 / kProducers;  // 16-byte chunks per producer / epilogue thread
  constexpr int S = Cfg::SLOTS;
  constexpr int K = Cfg::K;
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  // [B hi][B lo][staging images]; a staging image receives the raw tile (in
  // the A layout with cp.async, in natural tile order with a tensor copy), is
  // read by the converters, and with staged stores then carries the
  // accumulator back out.
  unsigned char* base_ptr = smem_dyn + ((1024 - (smem_u32(smem_dyn) & 1023)) & 1023);
  unsigned char* b_hi = base_ptr;
  unsigned char* b_lo = b_hi + Cfg::B_BYTES;
  unsigned char* raw = b_lo + Cfg::B_BYTES;

  constexpr int SB = Cfg::SB;
  constexpr int HS = Cfg::HSLOTS > 0 ? Cfg::HSLOTS : 1;
  __shared__ __align__(8) uint64_t bar_full[SB], bar_free[SB];
  __shared__ __align__(8) uint64_t bar_a_ready[2], bar_mma[2], bar_acc_free[2], bar_scale[kScaleRing];
  __shared__ uint32_t tmem_base_slot;
  // Tile bases, written by the producer when it issues a tile and read by
  // the epilogue once the tile's MMAs are done.  The producer runs at most
  // S + 4 tiles (k = 6 in halves: 6) ahead of the epilogue: it waits for a
  // slot that the converters free only after MMAs that wait for the
  // epilogue of two tiles back.  R entries cover that.
  constexpr int R = 2 * S > 8 ? 2 * S : 8;
  __shared__ uint64_t base_ring[R];
  // Per tile and TMEM lane: s + sb, the exponent the epilogue scales by.
  __shared__ int8_t row_exp[kScaleRing][128];
  __shared__ double norm_sh[4];
  __shared__ volatile int abort_flag;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    for (int i = 0; i < SB; ++i) {
      mbar_init(smem_u32(&bar_full[i]), g.tma_dims ? 1 : kProducers + 1);
      mbar_init(smem_u32(&bar_free[i]), g.direct ? kConverters : kEpilogue);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(smem_u32(&bar_a_ready[i]), kConverters);
      mbar_init(smem_u32(&bar_mma[i]), 1);
      mbar_init(smem_u32(&bar_acc_free[i]), kEpilogue);
    }
    for (int i = 0; i < kScaleRing; ++i) mbar_init(smem_u32(&bar_scale[i]), kConverters);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  {
    const uint4* src = reinterpret_cast<const uint4*>(bimg);
    uint4* dst = reinterpret_cast<uint4*>(b_hi);
    for (int i = tid; i < (2 * Cfg::B_BYTES) / 16; i += kTcThreads) dst[i] = src[i];
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
  const bool q0_group = !g.is_target[0];

  // Bounded wait; on timeout raise the flags and let every role leave.
  auto wait = [&](uint64_t* bar, uint32_t parity) -> bool {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < kWaitLimit; ++it) {
      uint32_t done;
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}"
          : "=r"(done)
          : "r"(a), "r"(parity)
          : "memory");
      if (done) return true;
      if ((it & 255) == 255 && abort_flag) return false;
    }
    abort_flag = 1;
    atomicExch(&g_tc_error, 1);
    return false;
  };
  auto arrive = [](uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
  };
  // Bounded drain of a copy's completion (no abort: the copy lands anyway).
  auto drain = [](uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < kWaitLimit; ++it) {
      uint32_t done;
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}"
          : "=r"(done)
          : "r"(a), "r"(parity)
          : "memory");
      if (done) return;
    }
  };

  // Chunk i of producer / epilogue thread t covers tile amplitudes
  // e = 2t + 256i and e + 1: amplitude e+1 sits at soff + 8 (qubit 0 is the
  // lowest target: next combination) or at soff + 8192 (qubit 0 is a group
  // bit: row + 64).  Offsets: this thread's (e = 2t) XOR the chunk table's.
  const uint32_t pair_step = q0_group ? 64u * 128u : 8u;
  auto pair_slot = [](int row, int comb) -> uint32_t { return pair_slot_offset(row, comb, DIM); };
  auto tile_base = [&](uint64_t t) -> uint64_t {
    uint64_t b = t << g.m_low;
    for (int j = 0; j < g.nh; ++j) {
      const int f = g.hpos[j];
      b = ((b >> f) << (f + 1)) | (b & ((uint64_t{1} << f) - 1));
    }
    return b;
  };

  if (warp < 4 && g.tma_dims) {
    // ------------------------------------------ producer, tensor-copy form
    // One thread fetches each tile with one tiled tensor copy (k = 6: two,
    // half q = 2j + h of tile j -- h the highest target's bit -- into slot
    // q % HS); an image holds its box in natural index order under the
    // 128-byte swizzle.
    if (tid == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmap)) : "memory");
      constexpr int PER = Cfg::HALVES ? 2 : 1;  // copies per tile
      constexpr int NS = Cfg::HALVES ? HS : S;
      constexpr uint32_t BYTES = Cfg::HALVES ? Cfg::HALF_BYTES : Cfg::RAW_BYTES;
      uint64_t issued = 0;
      for (uint64_t q = 0; q < PER * count; ++q) {
        const uint64_t j = q / PER;
        const int slot = (int)(q % NS);
        if (q >= (uint64_t)NS && !wait(&bar_free[slot], (uint32_t)(((q / NS) - 1) & 1))) break;
        uint64_t base = tile_base(first + j * stride);
        if (q % PER == 0) base_ring[j % R] = base;
        else base |= g.top_off;
        const uint32_t bar = smem_u32(&bar_full[slot]);
        mbar_arrive_expect_tx(bar, BYTES);
        int crd[5];
#pragma unroll
        for (int i = 0; i < 5; ++i) crd[i] = (int)((base >> g.tma_start[i]) & g.tma_mask[i]);
        tma_load_box(smem_u32(raw + slot * BYTES), &tmap, crd, g.tma_dims, bar);
        issued = q + 1;
      }
      // Drain: every issued copy lands before the CTA may leave (on the
      // normal path the converters have already seen them all).
      for (uint64_t q = issued > (uint64_t)NS ? issued - NS : 0; q < issued; ++q)
        drain(&bar_full[q % NS], (uint32_t)((q / NS) & 1));
    }
  } else if (warp < 4) {
    // ------------------------------------------------------------ producers
    uint64_t g0;
    uint32_t s0;
    amp_offsets(g, Cfg::TB, DIM, 2 * tid, false, &g0, &s0);
    for (uint64_t j = 0; j < count; ++j) {
      const int slot = (int)(j % S);
      if (j >= (uint64_t)S && !wait(&bar_free[slot], (uint32_t)(((j / S) - 1) & 1))) break;
      const uint64_t base = tile_base(first + j * stride);
      const uint32_t dst = smem_u32(raw + slot * Cfg::RAW_BYTES);
      const float2* src = s + base;
#pragma unroll
      for (int i = 0; i < CPT; ++i) {
        const uint64_t go = g0 ^ g.chunk_g[i];
        const uint32_t so = s0 ^ g.chunk_s_in[i];
        if (q0_group) {
          cp_async8(dst + so, src + go);
          cp_async8(dst + so + pair_step, src + go + 1);
        } else {
          cp_async16(dst + so, src + go);
        }
      }
      asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(&bar_full[slot]))
                   : "memory");
      if (tid == 0) {
        base_ring[j % R] = base;
        arrive(&bar_full[slot]);
      }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
  } else if (warp < 8) {
    // ----------------------------------------------------------- converters
    // Thread = A row (TMEM lane 32*(warp%4) + lane).  Per tile: the row's
    // largest magnitude m sets s (m * 2^s in [2^14, 2^15)); each element
    // x * 2^s splits into hi = fp16(x * 2^s), lo = fp16(x * 2^s - hi), two
    // fp16 per 32-bit column (re low, im high), into the A region of tile
    // parity j%2 once the MMAs of tile j-2 have released it; s + sb goes to
    // the epilogue through row_exp.
    // In the direct-store mode TMEM lane t carries group t (its cp.async
    // staging row is the rotated one); otherwise lane t carries staging row t.
    const int q = warp & 3;
    const int lane_row = 32 * q + lane;
    const int row = g.direct ? ((lane_row >> 1) | ((lane_row & 1) << (kGroupBits - 1))) : lane_row;
    const uint32_t lane_off = (uint32_t)(32 * q) << 16;
    const int sb = (int)bimg[2 * Cfg::B_BYTES / 4];
    // tensor-copy images: byte offset of this lane's group in the tile (or
    // in a half tile)
    uint32_t gtile = 0;
    if (Cfg::HALVES && g.tma_dims) {
#pragma unroll
      for (int b = 0; b < kGroupBits; ++b)
        if ((lane_row >> b) & 1) gtile |= g.gbit_off[b];
    } else {
      for (int jb = 0, gb = 0; jb < Cfg::TB; ++jb)
        if (!g.is_target[jb]) {
          if ((lane_row >> gb) & 1) gtile |= 8u << jb;
          ++gb;
        }
    }
    // The 128-byte swizzle (16-byte chunk c of 128-byte row r at c ^ (r mod
    // 8)) is linear over XOR, and group and target bits are disjoint, so an
    // amplitude's swizzled offset is the swizzled group offset XOR the
    // swizzled combination offset (ctile holds the latter).
    const uint32_t gsw = gtile ^ ((gtile >> 3) & 0x70u);
    // One loop per producer form, chosen once: with the form a compile-time
    // constant, every staging read of a tile has a constant offset and the
    // reads issue back to back (a per-read branch on the form kept only two
    // in flight, each paying the full shared-memory latency).
    auto convert_tiles = [&](auto form) {
      constexpr bool TMA = decltype(form)::value;
      constexpr bool HALF = TMA && Cfg::HALVES;
      for (uint64_t j = 0; j < count; ++j) {
        // the tile's images: one, or (k = 6 tensor copy) its two halves
        int slot0, slot1;
        bool ok;
        if constexpr (HALF) {
          slot0 = (int)((2 * j) % HS);
          slot1 = (int)((2 * j + 1) % HS);
          ok = wait(&bar_full[slot0], (uint32_t)(((2 * j) / HS) & 1)) &&
               wait(&bar_full[slot1], (uint32_t)(((2 * j + 1) / HS) & 1));
        } else {
          slot0 = slot1 = (int)(j % S);
          ok = wait(&bar_full[slot0], (uint32_t)((j / S) & 1));
        }
        // the A region is free once tile j-2's MMAs have completed
        if (!ok || (j >= 2 && !wait(&bar_mma[j & 1], (uint32_t)(((j - 2) >> 1) & 1)))) break;
        tc_fence_after();
        const unsigned char* img0 = raw + (HALF ? slot0 * Cfg::HALF_BYTES : slot0 * Cfg::RAW_BYTES);
        const unsigned char* img1 = raw + slot1 * Cfg::HALF_BYTES;
        // amplitudes 2i and 2i+1 of this row as (re, im, re, im)
        auto amp_pair = [&](int i) -> float4 {
          if constexpr (!TMA) {
            return *reinterpret_cast<const float4*>(img0 + sw128_offset(row, 4 * i, 128));
          } else {
            float2 v[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int c = 2 * i + h;
              const unsigned char* img = (HALF && c >= 32) ? img1 : img0;
              v[h] = *reinterpret_cast<const float2*>(img + (g.ctile[HALF ? (c & 31) : c] ^ gsw));
            }
            return make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
          }
        };
        // the row's largest magnitude, eight amplitude pairs per batch
        float m = 0.f;
#pragma unroll
        for (int bt = 0; bt < DIM / 16; ++bt) {
          float4 v[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) v[i] = amp_pair(8 * bt + i);
#pragma unroll
          for (int i = 0; i < 8; ++i)
            m = fmaxf(m, fmaxf(fmaxf(fabsf(v[i].x), fabsf(v[i].y)), fmaxf(fabsf(v[i].z), fabsf(v[i].w))));
        }
        // m in [2^e, 2^(e+1)) has exponent field e + 127; s = 14 - e, kept
        // within +-100 (a zero or subnormal row takes 100)
        const int ef = (int)(__float_as_uint(m) >> 23);
        const int sa = ef == 0 ? 100 : max(-100, min(100, 141 - ef));
        row_exp[j % kScaleRing][lane_row] = (int8_t)(sa + sb);
        arrive(&bar_scale[j % kScaleRing]);
        const float sc = __int_as_float((127 + sa) << 23);
        const f32x2 sc2 = pack2(sc, sc), neg1 = pack2(-1.f, -1.f);
        const uint32_t areg = tmem + lane_off + (uint32_t)((j & 1) * Cfg::A_COLS);
#pragma unroll
        for (int part = 0; part < K / 32; ++part) {
          uint32_t hi[16], lo[16];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const float4 v = amp_pair(8 * part + i);
            const f32x2 xs[2] = {mul_x2(pack2(v.x, v.y), sc2), mul_x2(pack2(v.z, v.w), sc2)};
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              const float2 x = unpack2(xs[u]);
              const __half2 h = __floats2half2_rn(x.x, x.y);
              const float2 hf = __half22float2(h);
              const float2 r = unpack2(fma_x2(pack2(hf.x, hf.y), neg1, xs[u]));  // x - hi, exact
              const __half2 l = __floats2half2_rn(r.x, r.y);
              hi[2 * i + u] = *reinterpret_cast<const uint32_t*>(&h);
              lo[2 * i + u] = *reinterpret_cast<const uint32_t*>(&l);
            }
          }
          tmem_st16(areg + (uint32_t)(part * 16), hi);
          tmem_st16(areg + (uint32_t)(K / 2 + part * 16), lo);
        }
        if (g.direct) {  // nothing else reads the images
          arrive(&bar_free[slot0]);
          if (slot1 != slot0) arrive(&bar_free[slot1]);
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        tc_fence_before();
        arrive(&bar_a_ready[j & 1]);
      }
    };
    if (g.tma_dims) convert_tiles(std::true_type{});
    else convert_tiles(std::false_type{});
  } else if (warp < 12) {
    // ------------------------------------------------------------- epilogue
    const int t = tid - 256;
    const int q = warp & 3;
    const int row = 32 * q + lane;
    const uint32_t acc_lane = tmem + (uint32_t)(2 * Cfg::A_COLS) + ((uint32_t)(32 * q) << 16);
    double nacc = 0.0;  // this thread's sum of |out|^2 (g.norm_out)
    // Waits for tile j's accumulator and row scale; returns 2^-(s + sb).
    auto tile_ready = [&](uint64_t j, float* unscale) -> bool {
      if (!wait(&bar_mma[j & 1], (uint32_t)((j >> 1) & 1))) return false;
      tc_fence_after();
      if (!wait(&bar_scale[j % kScaleRing], (uint32_t)((j / kScaleRing) & 1))) return false;
      *unscale = __int_as_float((127 - (int)row_exp[j % kScaleRing][row]) << 23);
      return true;
    };
    if (g.direct) {
      // TMEM lane = group `row`; the lanes of a warp vary the five lowest
      // group bits, which include qubits 0 and 1, so each run of lanes
      // fills whole 32-byte sectors.
      uint64_t gdep = 0;
      for (int jb = 0, gb = 0; jb < Cfg::TB; ++jb)
        if (!g.is_target[jb]) {
          if ((row >> gb) & 1) gdep |= uint64_t{1} << g.tile_pos[jb];
          ++gb;
        }
      for (uint64_t j = 0; j < count; ++j) {
        float us;
        if (!tile_ready(j, &us)) break;
        // tile j's base is in the ring once its MMAs are done (the
        // producer wrote it before the tile's copy was even issued)
        float2* dst = s + base_ring[j % R] + gdep;
        const f32x2 us2 = pack2(us, us);
        const uint32_t acc = acc_lane + (uint32_t)((j & 1) * N);
#pragma unroll
        for (int part = 0; part < N / 16; ++part) {
          float v[16];
          tmem_ld<16>(acc + (uint32_t)(part * 16), v);
          tmem_ld_wait();
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const float2 o = unpack2(mul_x2(pack2(v[2 * i], v[2 * i + 1]), us2));
            dst[g.cdep[part * 8 + i]] = o;
            if constexpr (NORM) nacc = fma((double)o.x, (double)o.x, fma((double)o.y, (double)o.y, nacc));
          }
        }
        tc_fence_before();
        arrive(&bar_acc_free[j & 1]);
      }
    } else {
      uint64_t g0;
      uint32_t s0;
      amp_offsets(g, Cfg::TB, DIM, 2 * t, true, &g0, &s0);
      for (uint64_t j = 0; j < count; ++j) {
        const int slot = (int)(j % S);
        unsigned char* out = raw + slot * Cfg::RAW_BYTES;
        float us;
        if (!tile_ready(j, &us)) break;
        const uint32_t acc = acc_lane + (uint32_t)((j & 1) * N);
#pragma unroll
        for (int part = 0; part < N / 16; ++part) {
          float v[16];
          tmem_ld<16>(acc + (uint32_t)(part * 16), v);
          tmem_ld_wait();
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            v[i] *= us;
            if constexpr (NORM) nacc = fma((double)v[i], (double)v[i], nacc);
          }
          if (q0_group) {
#pragma unroll
            for (int i = 0; i < 8; ++i)
              *reinterpret_cast<float2*>(out + pair_slot(row, part * 8 + i)) = make_float2(v[2 * i], v[2 * i + 1]);
          } else {
#pragma unroll
            for (int i = 0; i < 4; ++i)
              *reinterpret_cast<float4*>(out + sw128_offset(row, part * 16 + 4 * i, 128)) =
                  make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
          }
        }
        tc_fence_before();
        arrive(&bar_acc_free[j & 1]);
        asm volatile("bar.sync 1, %0;" ::"n"(kEpilogue) : "memory");
        float2* dst = s + base_ring[j % R];
#pragma unroll
        for (int i = 0; i < CPT; ++i)
          *reinterpret_cast<float4*>(dst + (g0 ^ g.chunk_g[i])) =
              *reinterpret_cast<const float4*>(out + (s0 ^ g.chunk_s_out[i]));
        arrive(&bar_free[slot]);
      }
    }
    if constexpr (NORM) {
      // the epilogue warps' sums, in a fixed order: warp, then warp 8..11
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) nacc += __shfl_xor_sync(0xffffffffu, nacc, o);
      if (lane == 0) norm_sh[q] = nacc;
      asm volatile("bar.sync 2, %0;" ::"n"(kEpilogue) : "memory");
      if (t == 0) g.norm_out[blockIdx.x] = (norm_sh[0] + norm_sh[1]) + (norm_sh[2] + norm_sh[3]);
    }
  } else if (warp == 12 && lane == 0) {
    // ------------------------------------------------------------ MMA issue
    constexpr uint32_t idesc = f16_idesc<N>();
    const uint32_t bh = smem_u32(b_hi), bl = smem_u32(b_lo);
    for (uint64_t j = 0; j < count; ++j) {
      if (!wait(&bar_a_ready[j & 1], (uint32_t)((j >> 1) & 1))) break;
      if (j >= 2 && !wait(&bar_acc_free[j & 1], (uint32_t)(((j >> 1) - 1) & 1))) break;
      tc_fence_after();
      const uint32_t ah = tmem + (uint32_t)((j & 1) * Cfg::A_COLS);
      const uint32_t al = ah + (uint32_t)(K / 2);
      const uint32_t acc = tmem + (uint32_t)(2 * Cfg::A_COLS + (j & 1) * N);
#pragma unroll
      for (int st = 0; st < Cfg::KSTEPS; ++st) {
        // K step st: 16 fp16 = 8 A columns; in B, 32 bytes of a 128-byte atom
        const uint32_t kbo = (uint32_t)((st >> 2) * N * 128 + (st & 3) * 32);
        tc_mma_f16_ts(acc, ah + 8 * st, sw128_desc(bh + kbo), idesc, st > 0 ? 1u : 0u);
        tc_mma_f16_ts(acc, ah + 8 * st, sw128_desc(bl + kbo), idesc, 1u);
        tc_mma_f16_ts(acc, al + 8 * st, sw128_desc(bh + kbo), idesc, 1u);
      }
      tc_commit(smem_u32(&bar_mma[j & 1]));
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(Cfg::TMEM_COLS)
                 : "memory");
  }
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

// Lowest target qubit from which a block always uses the tensor-copy
// producer (default 2: qubits 0 and 1 group bits).  A block whose lowest
// target is qubit 1 uses it when its converter reads stay conflict-free
// (tma_read_wavefronts).  KETGPU_TC_TMA=0 keeps every block on the cp.async
// producers, KETGPU_TC_TMA_MIN=q raises the threshold (for comparing the
// producer forms on one workload).
int tc_tma_min() {
  static const int v = [] {
    const char* e = std::getenv("KETGPU_TC_TMA");
    if (e && e[0] == '0') return 1 << 20;
    const char* m = std::getenv("KETGPU_TC_TMA_MIN");
    const int q = m ? std::atoi(m) : 2;
    return q < 0 ? 0 : q;
  }();
  return v;
}

// Tensor map over the state whose box is one tile: each dimension is a run
// of consecutive tile qubits followed by the non-tile qubits up to the next
// run, so a tile's coordinates are the non-tile bits of its base and the box
// lands in shared memory in the tile's natural index order, under the
// 128-byte swizzle.  The first dimension is qubits 0..3 (128 bytes, the
// swizzle's row); the others hold at most 8 tile qubits (the box limit of
// 256 elements); at most 5 dimensions.
//
// tile_runs (host only) returns the number of dimensions with each one's
// start qubit and tile-qubit count, or 0 when the tile breaks those limits.
int tile_runs(const TcGeom& g, int tb, int* start, int* tq) {
  int nd = 0;
  for (int j = 0; j < tb; ++j) {
    const int q = g.tile_pos[j];
    if (j == 0 || q != g.tile_pos[j - 1] + 1 || tq[nd - 1] == (nd == 1 ? 4 : 8)) {
      start[nd] = q;
      tq[nd] = 0;
      ++nd;
    }
    ++tq[nd - 1];
  }
  return (nd < 2 || nd > 5 || start[0] != 0 || tq[0] != 4) ? 0 : nd;
}

// Encodes the map for one launch and fills g's coordinate fields; returns
// the number of dimensions, or 0 (cp.async producers) when the tile breaks
// the limits or the driver has no encoder.
int encode_tile_map(const State& st, TcGeom& g, int tb, CUtensorMap* map) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return 0;
  int start[16], tq[16];
  const int nd = tile_runs(g, tb, start, tq);
  if (!nd) return 0;
  cuuint64_t dims[5], strides[4];
  cuuint32_t box[5], estr[5];
  for (int i = 0; i < nd; ++i) {
    const int end = i + 1 < nd ? start[i + 1] : st.n;
    dims[i] = cuuint64_t{1} << (end - start[i]);
    box[i] = 1u << tq[i];
    estr[i] = 1;
    if (i > 0) strides[i - 1] = (cuuint64_t{8}) << start[i];
    g.tma_start[i] = start[i];
    g.tma_mask[i] = dims[i] - 1;
  }
  for (int i = nd; i < 5; ++i) {
    g.tma_start[i] = 0;
    g.tma_mask[i] = 0;
  }
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, (cuuint32_t)nd, st.amps, dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? nd : 0;
}

int sm_count_tc(int device) {
  int v = 0;
  KB_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device));
  return v;
}

// Shared-memory wavefronts of the worst converter read of a tensor-copy tile
// (host only): lane l of converter warp q reads, for each combination c, the
// 8-byte amplitude of group 32q + l at its natural tile offset under the
// 128-byte swizzle.  A warp's 32 reads need at least 2 wavefronts; more
// means lanes whose groups lie 1 KB or more apart share banks.
int tma_read_wavefronts(const TcGeom& g, int tb, int dim) {
  int worst = 0;
  for (int q = 0; q < 4; ++q)
    for (int c = 0; c < dim; ++c) {
      uint32_t ctile = 0;
      for (int b = 0, jb = 0; jb < tb; ++jb)
        if (g.is_target[jb]) {
          if ((c >> b) & 1) ctile |= 8u << jb;
          ++b;
        }
      uint32_t words[32][2];
      for (int l = 0; l < 32; ++l) {
        const int lane_row = 32 * q + l;
        uint32_t gtile = 0;
        for (int jb = 0, gb = 0; jb < tb; ++jb)
          if (!g.is_target[jb]) {
            if ((lane_row >> gb) & 1) gtile |= 8u << jb;
            ++gb;
          }
        const uint32_t off = ctile | gtile;
        const uint32_t addr = off ^ ((off >> 3) & 0x70u);
        words[l][0] = addr >> 2;
        words[l][1] = (addr >> 2) + 1;
      }
      for (int bank = 0; bank < 32; ++bank) {
        uint32_t seen[64];
        int ns = 0;
        for (int l = 0; l < 32; ++l)
          for (int w = 0; w < 2; ++w)
            if ((words[l][w] & 31u) == (uint32_t)bank) {
              bool dup = false;
              for (int i = 0; i < ns; ++i) dup |= seen[i] == words[l][w];
              if (!dup) seen[ns++] = words[l][w];
            }
        worst = ns > worst ? ns : worst;
      }
    }
  return worst;
}

// Whether a block takes the tensor-copy producer (before the tile-run limits).
bool tma_wanted(const TcGeom& g, const Pass& p, int tb) {
  const int lowest = p.qubits[0];
  if (lowest >= tc_tma_min()) return true;
  return lowest == 1 && tc_tma_min() <= 2 && tma_read_wavefronts(g, tb, 1 << p.k) <= 2;
}

// Tile layout of a block on an n-qubit state (host only): the tile qubits,
// the tile index decomposition, each combination's offset and the
// cp.async-form direct-store rule.
template <int KQ>
void tile_geometry(int n, const Pass& p, TcGeom& g) {
  using Cfg = TcCfg<KQ>;
  g = TcGeom{};
  uint64_t tmask = 0;
  for (int b = 0; b < p.k; ++b) tmask |= uint64_t{1} << p.qubits[b];
  uint64_t tiles_mask = tmask;
  int extra = Cfg::TB - p.k;
  for (int q = 0; q < n && extra > 0; ++q)
    if (!((tmask >> q) & 1)) {
      tiles_mask |= uint64_t{1} << q;
      --extra;
    }
  if (extra > 0) fail(KETGPU_ERR_LOGIC, "tensor-core block needs n >= k + 7");
  int j = 0;
  for (int q = 0; q < n; ++q)
    if ((tiles_mask >> q) & 1) {
      g.tile_pos[j] = q;
      g.is_target[j] = (int)((tmask >> q) & 1);
      ++j;
    }
  g.m_low = 0;
  while (g.m_low < Cfg::TB && g.tile_pos[g.m_low] == g.m_low) ++g.m_low;
  // Direct stores from TMEM (lane t = group t) when qubit 0 is a group bit
  // and the five lowest group bits lie within qubits 0..5: a warp's 32
  // stores then fill 32-byte sectors within 512 contiguous bytes.  Otherwise
  // (qubit 0 a target, or the lanes spread thin) the output is staged
  // through shared memory and written in 16-byte words.  Blocks that take
  // the tensor-copy producer (qubits 0 and 1 group bits) store directly.
  {
    int seen = 0, fifth = 64;
    for (int b = 0; b < Cfg::TB && seen < 5; ++b)
      if (!g.is_target[b] && ++seen == 5) fifth = g.tile_pos[b];
    g.direct = (!g.is_target[0] && g.tile_pos[0] == 0 && fifth <= 5) ? 1 : 0;
  }
  for (int c = 0; c < (1 << p.k); ++c) {
    uint64_t d = 0;
    for (int b = 0; b < p.k; ++b)
      if ((c >> b) & 1) d |= uint64_t{1} << p.qubits[b];
    g.cdep[c] = d;
  }
  g.nh = 0;
  for (int i = g.m_low; i < Cfg::TB; ++i) g.hpos[g.nh++] = g.tile_pos[i];
  g.n_tiles = (uint64_t{1} << n) >> Cfg::TB;
  constexpr int CPT = Cfg::TILE / 2 / 128;
  static_assert(CPT <= 32, "chunk tables");
  for (int i = 0; i < CPT; ++i) {
    uint64_t go;
    uint32_t si, so;
    amp_offsets(g, Cfg::TB, Cfg::DIM, 256 * i, false, &go, &si);
    amp_offsets(g, Cfg::TB, Cfg::DIM, 256 * i, true, &go, &so);
    g.chunk_g[i] = go;
    g.chunk_s_in[i] = si;
    g.chunk_s_out[i] = so;
  }
}

// The half tile of a k = 6 block (host only): the tile less its highest
// target qubit `top`, as a 12-bit tile geometry.
void half_geometry(const TcGeom& g, int tb, int top, TcGeom& hg) {
  hg = g;
  int j = 0;
  for (int i = 0; i < tb; ++i)
    if (g.tile_pos[i] != top) {
      hg.tile_pos[j] = g.tile_pos[i];
      hg.is_target[j] = g.is_target[i];
      ++j;
    }
  for (; j < 16; ++j) hg.tile_pos[j] = hg.is_target[j] = 0;
}

// k = 6: whether the block takes the tensor copy in half tiles, and the
// half tiles' map, offsets and coordinates in g (host only).
int encode_half_tiles(const State* st, const Pass& p, TcGeom& g, CUtensorMap* map) {
  constexpr int TBH = 6 + kGroupBits - 1;
  TcGeom hg;
  half_geometry(g, TBH + 1, p.qubits[5], hg);
  Pass p5 = p;
  p5.k = 5;
  if (!tma_wanted(hg, p5, TBH)) return 0;
  int nd;
  if (st) {
    nd = encode_tile_map(*st, hg, TBH, map);
  } else {
    int start[16], tq[16];
    nd = tile_runs(hg, TBH, start, tq);
  }
  if (!nd) return 0;
  g.tma_dims = nd;
  g.half = 1;
  g.top_off = uint64_t{1} << p.qubits[5];
  g.direct = 1;
  for (int i = 0; i < 5; ++i) {
    g.tma_start[i] = hg.tma_start[i];
    g.tma_mask[i] = hg.tma_mask[i];
  }
  for (int c = 0; c < 32; ++c) {
    uint32_t off = 0;
    for (int b = 0, jb = 0; jb < TBH; ++jb)
      if (hg.is_target[jb]) {
        if ((c >> b) & 1) off |= 8u << jb;
        ++b;
      }
    g.ctile[c] = off ^ ((off >> 3) & 0x70u);  // swizzled (see the converters)
  }
  for (int b = 0, jb = 0; jb < TBH; ++jb)
    if (!hg.is_target[jb]) g.gbit_off[b++] = 8u << jb;
  return nd;
}

template <int KQ>
void launch_tc(const State& st, const Pass& p, const void* b_image, double* norm_partials) {
  using Cfg = TcCfg<KQ>;
  TcGeom g;
  tile_geometry<KQ>(st.n, p, g);
  g.norm_out = norm_partials;
  if (norm_partials)  // entries past the grid stay zero for the in-order sum
    KB_CUDA(cudaMemsetAsync(norm_partials, 0, sizeof(double) * kNormBlocks, st.stream));
  CUtensorMap tmap;
  std::memset(&tmap, 0, sizeof(tmap));
  // Tensor-copy blocks (qubit 0 a group bit) always store directly.
  if constexpr (KQ == 6) {
    g.tma_dims = encode_half_tiles(&st, p, g, &tmap);
  } else {
    g.tma_dims = tma_wanted(g, p, Cfg::TB) ? encode_tile_map(st, g, Cfg::TB, &tmap) : 0;
  }
  if (g.tma_dims && !g.half) {
    g.direct = 1;
    for (int c = 0; c < Cfg::DIM; ++c) {
      uint32_t off = 0;
      for (int b = 0, jb = 0; jb < Cfg::TB; ++jb)
        if (g.is_target[jb]) {
          if ((c >> b) & 1) off |= 8u << jb;
          ++b;
        }
      g.ctile[c] = off ^ ((off >> 3) & 0x70u);  // swizzled (see the converters)
    }
  }
  static int attr_done[64] = {0};
  if (st.device >= 0 && st.device < 64 && !(attr_done[st.device] & (1 << KQ))) {
    KB_CUDA(cudaFuncSetAttribute(fused_tc_kernel<KQ, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)Cfg::SMEM));
    KB_CUDA(cudaFuncSetAttribute(fused_tc_kernel<KQ, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)Cfg::SMEM));
    attr_done[st.device] |= 1 << KQ;
  }
  static int sms[64] = {0};
  if (!sms[st.device]) sms[st.device] = sm_count_tc(st.device);
  uint64_t grid = (uint64_t)sms[st.device];
  if (grid > g.n_tiles) grid = g.n_tiles;
  if (norm_partials && grid > (uint64_t)kNormBlocks) fail(KETGPU_ERR_LOGIC, "tensor-core norm partials");
  if (norm_partials)
    fused_tc_kernel<KQ, true><<<(unsigned)grid, kTcThreads, Cfg::SMEM, st.stream>>>(
        static_cast<float2*>(st.amps), g, static_cast<const uint32_t*>(b_image), tmap);
  else
    fused_tc_kernel<KQ, false><<<(unsigned)grid, kTcThreads, Cfg::SMEM, st.stream>>>(
        static_cast<float2*>(st.amps), g, static_cast<const uint32_t*>(b_image), tmap);
  count_launch();
  KB_CUDA(cudaGetLastError());
}

// IEEE binary16 bits of v, rounded to nearest, ties to even (host only), by
// integer operations on the double's fields: keep the top 11 significant
// bits (fewer below 2^-14, where the spacing is 2^-24), round on the bits
// dropped, and let a carry move the exponent.
uint16_t host_f16_bits(double v) {
  uint64_t b;
  std::memcpy(&b, &v, 8);
  const uint16_t sign = (uint16_t)((b >> 48) & 0x8000u);
  b &= 0x7fffffffffffffffull;
  if (b > 0x7ff0000000000000ull) return (uint16_t)(sign | 0x7e00u);  // NaN
  const int e = (int)(b >> 52) - 1023;  // v in [2^e, 2^(e+1)) for normal doubles
  if (e > 15) return (uint16_t)(sign | 0x7c00u);  // 2^16 and up, infinity
  if (e < -25) return sign;                        // below half the least subnormal
  const uint64_t m = (b & ((uint64_t{1} << 52) - 1)) | (uint64_t{1} << 52);  // 53-bit significand
  const int shift = e >= -14 ? 42 : 42 + (-14 - e);  // bits dropped
  uint64_t q = m >> shift;
  const uint64_t rem = m & ((uint64_t{1} << shift) - 1), half = uint64_t{1} << (shift - 1);
  if (rem > half || (rem == half && (q & 1))) ++q;
  if (e < -14) return (uint16_t)(sign | q);  // subnormal (q = 1024: the least normal)
  int E = e;
  if (q == 2048) {
    q = 1024;
    ++E;
  }
  if (E > 15) return (uint16_t)(sign | 0x7c00u);
  return (uint16_t)(sign | ((E + 15) << 10) | (q - 1024));
}

double host_f16_value(uint16_t h) {
  const int ex = (h >> 10) & 31, man = h & 1023;
  double v;
  if (ex == 0) {
    v = man * 5.9604644775390625e-08;  // man * 2^-24, exact
  } else {
    const uint64_t bits = ((uint64_t)(ex - 15 + 1023) << 52) | ((uint64_t)man << 42);
    std::memcpy(&v, &bits, 8);
  }
  return (h & 0x8000u) ? -v : v;
}

}  // namespace

bool tc_supported(int k) { return k >= 4 && k <= 6; }

// hi and lo images of whole 128-byte atoms along K, then the scale word
size_t tc_image_bytes(int k) {
  const size_t dim = size_t{1} << k;
  return 2 * ((2 * dim + 63) / 64) * (2 * dim) * 128 + 16;
}

// B = real embedding of mat (row-major dim x dim complex) scaled by 2^sb
// (its largest entry into [2^14, 2^15)), stored as the K-major SW128 fp16
// images hi then lo (N rows of K halves each), then sb as a 32-bit integer.
void build_tc_image(const std::vector<cplx>& mat, int k, std::vector<uint32_t>& out) {
  const int dim = 1 << k, K = 2 * dim, N = 2 * dim;
  out.assign(tc_image_bytes(k) / 4, 0u);
  double maxb = 0;
  for (const cplx& m : mat) maxb = std::max(maxb, std::max(std::fabs(m.real()), std::fabs(m.imag())));
  int sb = 14;
  if (maxb > 0) {
    int ex;
    std::frexp(maxb, &ex);  // maxb in [2^(ex-1), 2^ex)
    sb = std::max(-24, std::min(24, 15 - ex));
  }
  const size_t img = (tc_image_bytes(k) - 16) / 2;
  unsigned char* hi = reinterpret_cast<unsigned char*>(out.data());
  unsigned char* lo = hi + img;
  const double scale = std::ldexp(1.0, sb);  // a power of two: exact products
  for (int n = 0; n < N; ++n)
    for (int kk = 0; kk < K; ++kk) {
      const int r = n >> 1, c = kk >> 1;
      const cplx m = mat[(size_t)r * dim + c];
      double v;
      if ((n & 1) == 0) v = (kk & 1) == 0 ? m.real() : -m.imag();
      else v = (kk & 1) == 0 ? m.imag() : m.real();
      v *= scale;
      const uint16_t h = host_f16_bits(v);
      const uint16_t l = host_f16_bits(v - host_f16_value(h));
      const uint32_t off = sw128_offset_h(n, kk, N);
      if (off + 2 > img) fail(KETGPU_ERR_LOGIC, "tensor-core image layout");
      std::memcpy(hi + off, &h, 2);
      std::memcpy(lo + off, &l, 2);
    }
  const int32_t sbw = sb;
  std::memcpy(lo + img, &sbw, 4);
}

void launch_fused_tc(const State& s, const Pass& p, const void* b_image, double* norm_partials) {
  if (p.k == 5) launch_tc<5>(s, p, b_image, norm_partials);
  else if (p.k == 4) launch_tc<4>(s, p, b_image, norm_partials);
  else if (p.k == 6) launch_tc<6>(s, p, b_image, norm_partials);
  else fail(KETGPU_ERR_LOGIC, "tensor-core block supports k = 4, 5 or 6");
}

void tc_form(int n, const Pass& p, int* tma_dims, int* direct) {
  if (p.k < 4 || p.k > 6) fail(KETGPU_ERR_LOGIC, "tensor-core block supports k = 4, 5 or 6");
  TcGeom g;
  if (p.k == 5) tile_geometry<5>(n, p, g);
  else if (p.k == 6) tile_geometry<6>(n, p, g);
  else tile_geometry<4>(n, p, g);
  int start[16], tq[16];
  const int nd = p.k == 6 ? encode_half_tiles(nullptr, p, g, nullptr)
                 : tma_wanted(g, p, p.k + kGroupBits) ? tile_runs(g, p.k + kGroupBits, start, tq)
                                                       : 0;
  *tma_dims = nd;
  *direct = nd ? 1 : g.direct;
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
