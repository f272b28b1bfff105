// adj_tile.cuh -- device code of the tiled adjoint sweeps shared by the
// kernels compiled with the library (adjoint.cu) and by the per-block
// complex64 kernels that adjoint.cu generates and compiles at run time
// (NVRTC; the build embeds this file's text).  Under NVRTC (KB_JIT) no host
// headers are available, so the fixed-width integer types are declared here.
#pragma once
#ifdef KB_JIT
typedef unsigned long long uint64_t;
typedef unsigned int uint32_t;
typedef unsigned short uint16_t;
typedef unsigned char uint8_t;
typedef long long int64_t;
typedef int int32_t;
typedef short int16_t;
typedef signed char int8_t;
#else
#include <cuda_runtime.h>

#include <cstdint>
#endif

namespace kbt {

template <typename R>
struct TileCfg;
template <>
struct TileCfg<float> {
  static constexpr int TB = 12, RB = 4;
};
template <>
struct TileCfg<double> {
  static constexpr int TB = 11, RB = 3;
};
constexpr int kTileThreads = 256;  // 2^(TB - RB) in both precisions
constexpr int kTileWarps = kTileThreads / 32;
constexpr int kMaxBlockGrads = 64;
constexpr int kMaxBlockGates = 256;

enum TKind : uint8_t { kTPair = 0, kTPairSwap = 1, kTSwap2 = 2, kTDiag = 3 };

struct TGate {
  uint8_t kind;
  uint8_t s0, s1;  // register slots of the target(s) (pair kinds; s0 < s1 for kTSwap2)
  int8_t tslot;    // kTDiag: register slot of the target bit, or -1
  uint8_t tbit;    // kTDiag: tile bit of the target
  uint8_t cm_r;    // controls held in registers, as a register-index mask
  uint8_t gen;     // gradient generator: 0 none, 1 X, 2 Y, 3 Z, 4 P11
  uint8_t real;    // kTPair: the matrix is real for every parameter set
  uint16_t cm_g;   // controls not held in registers, as a tile-bit mask
  int16_t grad;    // gradient slot within the block, or -1
  int32_t mat;     // gate index into the per-set matrix table
};
static_assert(sizeof(TGate) == 16, "TGate layout");

struct TPhase {
  uint8_t r[4];  // tile bits held in registers (register-index bit b <-> r[b])
  int32_t first, count;  // gates of the phase, relative to the block's first gate
};

struct TileGeom {
  uint64_t n_tiles;
  int pos[12];  // tile bit -> qubit, ascending; pos[0..4] = 0..4
};

// Shared-memory swizzle: XOR-folds the higher bit groups into the lowest so
// that a half-warp (8-byte elements) or quarter-warp (16-byte elements)
// touching 16 (8) elements that differ in any four (three) tile bits hits
// distinct banks in the common layouts.
template <typename R>
__device__ __forceinline__ int tphys(int e);
template <>
__device__ __forceinline__ int tphys<float>(int e) {
  return e ^ (((e >> 4) ^ (e >> 8)) & 15);
}
template <>
__device__ __forceinline__ int tphys<double>(int e) {
  return e ^ (((e >> 3) ^ (e >> 6) ^ (e >> 9)) & 7);
}


// Asynchronous global -> shared copy of one amplitude (8 or 16 bytes).
__device__ __forceinline__ void tile_cp_async(float2* dst, const float2* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void tile_cp_async(double2* dst, const double2* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

// ---------------------------------------------------------------------------
// complex64 tiled sweeps on packed pairs.  Blackwell's f32x2 instructions
// (fma.rn.f32x2, mul.rn.f32x2) do two FP32 operations each.  Register slot 0 of a
// complex64 phase is its pack bit: no gate of the phase targets it with a
// pair or uses it as a control (the planner guarantees it), so the two
// amplitudes that differ only in that bit always meet the same coefficients
// and live in one 64-bit register pair: re = (re_lo, re_hi), im = (im_lo,
// im_hi).  A thread's 16 amplitudes of a state are 8 such packs of each
// part; a gate on register slot S (1..3) acts across packs jo and
// jo | 1 << (S-1).  A diagonal gate may target the pack bit itself (its two
// phases then form a per-half pack).  Per gate the shared memory holds 16
// packed coefficients of U (forward) or U^dag (reverse):
//   [0..7]  c0r c0i c1r c1i c2r c2i c3r c3i, each duplicated in both halves
//   [8..11] -c0i -c1i -c2i -c3i
//   [12..14] (c0r, c3r) (c0i, c3i) (-c0i, -c3i): a diagonal on the pack bit
using f2 = unsigned long long;  // (lo, hi) halves in one 64-bit register pair

__device__ __forceinline__ f2 pk2(float lo, float hi) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void upk2(f2 v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
  f2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ f2 mul2p(f2 a, f2 b) {
  f2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ float hsum2(f2 v) {
  float lo, hi;
  upk2(v, lo, hi);
  return lo + hi;
}

struct PackState {
  f2 r[8], i[8];
};

// (xr, xi) <- complex phase (pr, pi) times (xr, xi); npi = -pi.
__device__ __forceinline__ void pk_phase(f2& xr, f2& xi, f2 pr, f2 pi, f2 npi) {
  const f2 nr = fma2(pr, xr, mul2p(npi, xi));
  xi = fma2(pr, xi, mul2p(pi, xr));
  xr = nr;
}

// 2x2 on packs a, b: (a, b) <- (c0 a + c1 b, c2 a + c3 b).
template <bool REAL>
__device__ __forceinline__ void pk_2x2(f2& ar, f2& ai, f2& br, f2& bi, const f2* c) {
  if (REAL) {
    const f2 xr = fma2(c[0], ar, mul2p(c[2], br)), xi = fma2(c[0], ai, mul2p(c[2], bi));
    const f2 yr = fma2(c[4], ar, mul2p(c[6], br)), yi = fma2(c[4], ai, mul2p(c[6], bi));
    ar = xr, ai = xi, br = yr, bi = yi;
  } else {
    const f2 xr = fma2(c[0], ar, fma2(c[8], ai, fma2(c[2], br, mul2p(c[9], bi))));
    const f2 xi = fma2(c[0], ai, fma2(c[1], ar, fma2(c[2], bi, mul2p(c[3], br))));
    const f2 yr = fma2(c[4], ar, fma2(c[10], ai, fma2(c[6], br, mul2p(c[11], bi))));
    const f2 yi = fma2(c[4], ai, fma2(c[5], ar, fma2(c[6], bi, mul2p(c[7], br))));
    ar = xr, ai = xi, br = yr, bi = yi;
  }
}

// Gate bodies, fully specialised at compile time: register slot(s), real or
// complex matrix, gradient generator (reverse only) and whether some
// controls are register bits (RC; then each pack is tested against them).

// Swap on outer slot S (1..3): X, CX, CCX.
template <int S, bool REV, bool RC>
__device__ __forceinline__ float pk_swap(PackState& a, PackState& l, const TGate& g) {
  constexpr int so = S - 1;
  const int cm = g.cm_r >> 1;
#pragma unroll
  for (int jo = 0; jo < 8; ++jo) {
    if (jo & (1 << so)) continue;
    if (RC && (jo & cm) != cm) continue;
    const int j1 = jo | (1 << so);
    f2 t = a.r[jo]; a.r[jo] = a.r[j1]; a.r[j1] = t;
    t = a.i[jo]; a.i[jo] = a.i[j1]; a.i[j1] = t;
    if (REV) {
      t = l.r[jo]; l.r[jo] = l.r[j1]; l.r[j1] = t;
      t = l.i[jo]; l.i[jo] = l.i[j1]; l.i[j1] = t;
    }
  }
  return 0.f;
}

// 2x2 on outer slot S.  Reverse: the gradient term Im <l|G|a> first (GEN
// 1 X, 2 Y, 3 Z), as plus and minus packed sums.
template <int S, bool REAL, int GEN, bool REV, bool RC>
__device__ __forceinline__ float pk_pair(PackState& a, PackState& l, const TGate& g, const f2* c) {
  constexpr int so = S - 1;
  const int cm = g.cm_r >> 1;
  f2 plus = 0, minus = 0;
#pragma unroll
  for (int jo = 0; jo < 8; ++jo) {
    if (jo & (1 << so)) continue;
    if (RC && (jo & cm) != cm) continue;
    const int j1 = jo | (1 << so);
    if (REV && GEN == 1) {  // X: (l0r a1i - l0i a1r) + (l1r a0i - l1i a0r)
      plus = fma2(l.r[jo], a.i[j1], fma2(l.r[j1], a.i[jo], plus));
      minus = fma2(l.i[jo], a.r[j1], fma2(l.i[j1], a.r[jo], minus));
    } else if (REV && GEN == 2) {  // Y: (l1r a0r + l1i a0i) - (l0r a1r + l0i a1i)
      plus = fma2(l.r[j1], a.r[jo], fma2(l.i[j1], a.i[jo], plus));
      minus = fma2(l.r[jo], a.r[j1], fma2(l.i[jo], a.i[j1], minus));
    } else if (REV && GEN == 3) {  // Z: (l0r a0i - l0i a0r) - (l1r a1i - l1i a1r)
      plus = fma2(l.r[jo], a.i[jo], fma2(l.i[j1], a.r[j1], plus));
      minus = fma2(l.i[jo], a.r[jo], fma2(l.r[j1], a.i[j1], minus));
    }
    pk_2x2<REAL>(a.r[jo], a.i[jo], a.r[j1], a.i[j1], c);
    if (REV) pk_2x2<REAL>(l.r[jo], l.i[jo], l.r[j1], l.i[j1], c);
  }
  return (REV && GEN) ? hsum2(plus) - hsum2(minus) : 0.f;
}

template <int A, int B, bool REV, bool RC>
__device__ __forceinline__ float pk_swap2(PackState& a, PackState& l, const TGate& g) {
  constexpr int oa = A - 1, ob = B - 1;
  const int cm = g.cm_r >> 1;
#pragma unroll
  for (int jo = 0; jo < 8; ++jo) {
    if (!(jo & (1 << oa)) || (jo & (1 << ob))) continue;
    if (RC && (jo & cm) != cm) continue;
    const int j1 = jo ^ (1 << oa) ^ (1 << ob);
    f2 t = a.r[jo]; a.r[jo] = a.r[j1]; a.r[j1] = t;
    t = a.i[jo]; a.i[jo] = a.i[j1]; a.i[j1] = t;
    if (REV) {
      t = l.r[jo]; l.r[jo] = l.r[j1]; l.r[j1] = t;
      t = l.i[jo]; l.i[jo] = l.i[j1]; l.i[j1] = t;
    }
  }
  return 0.f;
}

// Diagonal gate.  TS: register slot of the target (1..3), 0 for the pack
// bit, -1 for a group bit (its value for this thread is read from gbase).
// Gradient (GEN 3 Z, 4 P11): Im(conj(l) a) per amplitude, weighted +-1 by the
// target bit (Z) or kept only where it is 1 (P11).
template <int TS, int GEN, bool REV, bool RC>
__device__ __forceinline__ float pk_diag(PackState& a, PackState& l, const TGate& g, const f2* c, int gbase) {
  const int cm = g.cm_r >> 1;
  const bool gbit = TS < 0 ? ((gbase >> g.tbit) & 1) : false;
  f2 plus0 = 0, minus0 = 0, plus1 = 0, minus1 = 0;  // target bit 0 / 1
  f2 pr0 = c[0], pi0 = c[1], npi0 = c[8], pr1 = c[6], pi1 = c[7], npi1 = c[11];
  if (TS == 0) pr0 = c[12], pi0 = c[13], npi0 = c[14];
  if (TS < 0 && gbit) pr0 = pr1, pi0 = pi1, npi0 = npi1;
#pragma unroll
  for (int jo = 0; jo < 8; ++jo) {
    if (RC && (jo & cm) != cm) continue;
    const bool bit = TS > 0 ? ((jo >> (TS - 1)) & 1) : false;  // compile time
    const f2 pr = bit ? pr1 : pr0, pi = bit ? pi1 : pi0, npi = bit ? npi1 : npi0;
    if (REV && GEN) {
      if (!bit) {
        plus0 = fma2(l.r[jo], a.i[jo], plus0);
        minus0 = fma2(l.i[jo], a.r[jo], minus0);
      } else {
        plus1 = fma2(l.r[jo], a.i[jo], plus1);
        minus1 = fma2(l.i[jo], a.r[jo], minus1);
      }
    }
    pk_phase(a.r[jo], a.i[jo], pr, pi, npi);
    if (REV) pk_phase(l.r[jo], l.i[jo], pr, pi, npi);
  }
  if (!(REV && GEN)) return 0.f;
  float s0, s1;
  if (TS == 0) {  // halves: lo = target bit 0, hi = target bit 1
    float p0, p1, m0, m1;
    upk2(plus0, p0, p1);
    upk2(minus0, m0, m1);
    s0 = p0 - m0;
    s1 = p1 - m1;
  } else if (TS < 0) {  // every element of the thread has target bit gbit
    const float t = hsum2(plus0) - hsum2(minus0);
    s0 = gbit ? 0.f : t;
    s1 = gbit ? t : 0.f;
  } else {
    s0 = hsum2(plus0) - hsum2(minus0);
    s1 = hsum2(plus1) - hsum2(minus1);
  }
  return GEN == 3 ? s0 - s1 : s1;
}

// Flat opcode of a gate, computed once per CTA when the block's gates are
// staged (the generator counts only in the reverse sweep):
//   pair   (S-1)*16 + real*8 + gen*2 + rc           0..47
//   swap   48 + (S-1)*2 + rc                         48..53
//   swap2  54 + {(1,2):0, (1,3):1, (2,3):2}*2 + rc   54..59
//   diag   60 + (TS+1)*6 + {0:0, 3:1, 4:2}[gen]*2 + rc   60..89
__device__ __forceinline__ int pk_opcode(const TGate& g, bool rev) {
  const int rc = g.cm_r ? 1 : 0;
  const int gen = rev ? g.gen : 0;
  switch (g.kind) {
    case kTPair: return (g.s0 - 1) * 16 + (g.real ? 8 : 0) + gen * 2 + rc;
    case kTPairSwap: return 48 + (g.s0 - 1) * 2 + rc;
    case kTSwap2: return 54 + (g.s0 == 1 ? (g.s1 == 2 ? 0 : 1) : 2) * 2 + rc;
    default: return 60 + (g.tslot + 1) * 6 + (gen == 3 ? 1 : gen == 4 ? 2 : 0) * 2 + rc;
  }
}

template <int OP, bool REV>
__device__ __forceinline__ float pk_exec(PackState& a, PackState& l, const TGate& g, const f2* c, int gbase) {
  if constexpr (OP < 48) {
    return pk_pair<OP / 16 + 1, ((OP / 8) & 1) != 0, (OP / 2) & 3, REV, (OP & 1) != 0>(a, l, g, c);
  } else if constexpr (OP < 54) {
    return pk_swap<(OP - 48) / 2 + 1, REV, (OP & 1) != 0>(a, l, g);
  } else if constexpr (OP < 60) {
    constexpr int w = (OP - 54) / 2;
    return pk_swap2<w == 2 ? 2 : 1, w == 0 ? 2 : 3, REV, (OP & 1) != 0>(a, l, g);
  } else {
    constexpr int t = (OP - 60) / 6, gi = ((OP - 60) % 6) / 2;
    return pk_diag<t - 1, gi == 0 ? 0 : gi == 1 ? 3 : 4, REV, (OP & 1) != 0>(a, l, g, c, gbase);
  }
}

#define KB_PK_CASE(N) \
  case N: return pk_exec<N, REV>(a, l, g, c, gbase);
#define KB_PK_CASE10(N)                                                                                    \
  KB_PK_CASE(N + 0) KB_PK_CASE(N + 1) KB_PK_CASE(N + 2) KB_PK_CASE(N + 3) KB_PK_CASE(N + 4) KB_PK_CASE(N + 5) \
  KB_PK_CASE(N + 6) KB_PK_CASE(N + 7) KB_PK_CASE(N + 8) KB_PK_CASE(N + 9)

template <bool REV>
__device__ __forceinline__ float pk_dispatch(int op, PackState& a, PackState& l, const TGate& g, const f2* c,
                                             int gbase) {
  switch (op) {
    KB_PK_CASE10(0) KB_PK_CASE10(10) KB_PK_CASE10(20) KB_PK_CASE10(30) KB_PK_CASE10(40)
    KB_PK_CASE10(50) KB_PK_CASE10(60) KB_PK_CASE10(70) KB_PK_CASE10(80)
    default: return 0.f;
  }
}
#undef KB_PK_CASE10
#undef KB_PK_CASE

// ---------------------------------------------------------------------------
// Pieces of a complex64 tiled sweep, used by the per-block kernels that are
// generated with their phases and gates as compile-time constants.

// Per-CTA set-up: tile offset tables, the block's gate records and this
// set's packed coefficients (U forward, U^dag reverse), and `acc_words`
// zeroed 4-byte words of gradient sums.
template <bool REV>
__device__ __forceinline__ void c64_setup(const TileGeom& tg, const TGate* __restrict__ gates, int ngates,
                                          const float* __restrict__ mats, uint64_t mat_stride, int set,
                                          int acc_words, uint64_t* off_lo, uint64_t* off_hi, f2* spk,
                                          float* acc) {
  constexpr int TB = TileCfg<float>::TB;
  const int tid = threadIdx.x;
  if (tid < 128) {
    const int half = tid >> 6, e = tid & 63;
    uint64_t off = 0;
    for (int b = 0; b < 6; ++b) {
      const int tb = 6 * half + b;
      if (tb < TB && ((e >> b) & 1)) off |= (uint64_t)1 << tg.pos[tb];
    }
    (half ? off_hi : off_lo)[e] = off;
  }
  for (int i = tid; i < ngates; i += kTileThreads) {
    const float* m = mats + ((uint64_t)gates[i].mat * mat_stride + set) * 8;
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
    for (int i = tid; i < acc_words; i += kTileThreads) acc[i] = 0.f;
}

__device__ __forceinline__ uint64_t c64_tile_base(const TileGeom& tg, uint64_t t) {
  uint64_t base = t;
#pragma unroll
  for (int b = 0; b < TileCfg<float>::TB; ++b) {
    const int f = tg.pos[b];
    base = ((base >> f) << (f + 1)) | (base & (((uint64_t)1 << f) - 1));
  }
  return base;
}

template <bool REV>
__device__ __forceinline__ void c64_prefetch(const TileGeom& tg, const uint64_t* off_lo, const uint64_t* off_hi,
                                             uint64_t t, float2* buf, const float2* s, const float2* l) {
  constexpr int TILE = 1 << TileCfg<float>::TB;
  const uint64_t base = c64_tile_base(tg, t);
#pragma unroll 2
  for (int r = 0; r < 16; ++r) {
    const int e = threadIdx.x + r * kTileThreads;
    const uint64_t o = base + (off_lo[e & 63] | off_hi[e >> 6]);
    tile_cp_async(buf + tphys<float>(e), s + o);
    if (REV) tile_cp_async(buf + TILE + tphys<float>(e), l + o);
  }
}

template <bool REV>
__device__ __forceinline__ void c64_store_tile(const TileGeom& tg, const uint64_t* off_lo, const uint64_t* off_hi,
                                               uint64_t t, const float2* sp, const float2* sl, float2* s, float2* l) {
  const uint64_t base = c64_tile_base(tg, t);
  const volatile uint64_t* vlo = off_lo;
  const volatile uint64_t* vhi = off_hi;
#pragma unroll 2
  for (int r = 0; r < 16; ++r) {
    const int e = threadIdx.x + r * kTileThreads;
    const uint64_t o = base + (vlo[e & 63] | vhi[e >> 6]);
    s[o] = sp[tphys<float>(e)];
    if (REV) l[o] = sl[tphys<float>(e)];
  }
}

// Shared-memory addresses of pack jo: pg ^ (pb1, pb2, pb3 by the bits of jo),
// and the same ^ pb0 for its upper half.
template <bool REV>
__device__ __forceinline__ void c64_load_phase(const float2* sp, const float2* sl, int pg, int pb0, int pb1, int pb2,
                                               int pb3, PackState& A, PackState& L) {
#pragma unroll
  for (int jo = 0; jo < 8; ++jo) {
    const int a0 = pg ^ ((jo & 1) ? pb1 : 0) ^ ((jo & 2) ? pb2 : 0) ^ ((jo & 4) ? pb3 : 0);
    const int a1 = a0 ^ pb0;
    const float2 x = sp[a0], y = sp[a1];
    A.r[jo] = pk2(x.x, y.x);
    A.i[jo] = pk2(x.y, y.y);
    if (REV) {
      const float2 u = sl[a0], v = sl[a1];
      L.r[jo] = pk2(u.x, v.x);
      L.i[jo] = pk2(u.y, v.y);
    }
  }
}

template <bool REV>
__device__ __forceinline__ void c64_store_phase(float2* sp, float2* sl, int pg, int pb0, int pb1, int pb2, int pb3,
                                                const PackState& A, const PackState& L) {
#pragma unroll
  for (int jo = 0; jo < 8; ++jo) {
    const int a0 = pg ^ ((jo & 1) ? pb1 : 0) ^ ((jo & 2) ? pb2 : 0) ^ ((jo & 4) ? pb3 : 0);
    const int a1 = a0 ^ pb0;
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

// Warp sum of a gradient term (FP64) into the warp's slot.
__device__ __forceinline__ void c64_grad(double* acc, int ngrad, int slot, float part) {
  double v = (double)part;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) acc[(threadIdx.x >> 5) * ngrad + slot] += v;
}

__device__ __forceinline__ void c64_flush(const double* acc, int ngrad, double* partial, int set) {
  for (int g = threadIdx.x; g < ngrad; g += kTileThreads) {
    double v = 0.0;
    for (int w = 0; w < kTileWarps; ++w) v += acc[w * ngrad + g];
    partial[((uint64_t)set * ngrad + g) * gridDim.x + blockIdx.x] = v;
  }
}

// Blocks with few gradients: each thread sums its own gradient terms over
// all of its tiles in FP32, in shared-memory slots of stride GS (odd, so a
// warp's slots fall in distinct banks), with no per-tile warp reduction.
// The CTA folds the slots in FP64, in thread order, once at its end.
__device__ __forceinline__ void c64_grad_slot(float* accf, int gs, int slot, float part) {
  accf[threadIdx.x * gs + slot] += part;
}

__device__ __forceinline__ void c64_flush_slots(const float* accf, int gs, int ngrad, double* partial, int set) {
  for (int g = threadIdx.x; g < ngrad; g += kTileThreads) {
    double v = 0.0;
    for (int t = 0; t < kTileThreads; ++t) v += (double)accf[t * gs + g];
    partial[((uint64_t)set * ngrad + g) * gridDim.x + blockIdx.x] = v;
  }
}

}  // namespace kbt
