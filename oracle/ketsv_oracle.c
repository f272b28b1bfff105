/*
 * ketsv_oracle.c -- CPU oracle for the ket state-vector path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  A plain-C
 * restatement of the reference's complex128 algorithm:
 *   - per-gate loops            src/simulator.cpp:23-254
 *   - gate dispatch             src/simulator.cpp:259-338
 *   - dense m-qubit apply       src/simulator.cpp:357-393
 *   - greedy Fuser              src/simulator.cpp:400-477
 *   - circuit driver / run      src/simulator.cpp:482-558
 *   - Pauli expectation         src/observable.cpp:18-91
 *   - Born-rule measure         src/measurement.cpp:12-21
 * Complex products are written out as (ac - bd, ad + bc), the expansion GCC
 * emits for std::complex<double>::operator*, and the file is compiled with
 * -ffp-contract=off so no multiply-add is fused; per-gate results therefore
 * agree bit for bit with ket::run built by the same compiler.
 *
 * The fixed-tree sampler, the adjoint gradient and the MLP reference have no
 * counterpart in the reference; each is restated from its mathematics below.
 */
#include "ketsv_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  double re, im;
} cx;

static inline cx C(double re, double im) {
  cx z;
  z.re = re;
  z.im = im;
  return z;
}
static inline cx cmul(cx a, cx b) {
  return C(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
static inline cx cadd(cx a, cx b) { return C(a.re + b.re, a.im + b.im); }
static inline cx csub(cx a, cx b) { return C(a.re - b.re, a.im - b.im); }
static inline cx cscale(cx a, double s) { return C(a.re * s, a.im * s); }
static inline cx cneg(cx a) { return C(-a.re, -a.im); }
static inline cx cconj(cx a) { return C(a.re, -a.im); }
/* std::polar(rho, theta) in libstdc++: (rho*cos(theta), rho*sin(theta)). */
static inline cx cpolar(double rho, double th) {
  return C(rho * cos(th), rho * sin(th));
}

#define AMP(s, k) (((cx*)(s))[(k)])

/* ---------------------------------------------------------------------------
 * Per-gate loops (simulator.cpp:23-254).  `s` is the interleaved array; each
 * loop visits the owner index (the one with the moving bit(s) cleared). */

static void apply_single(double* s, size_t dim, int q, cx m00, cx m01, cx m10,
                         cx m11) {
  const size_t mask = (size_t)1 << q;
  for (size_t k = 0; k < dim; ++k) {
    if (k & mask) continue;
    const size_t k1 = k | mask;
    const cx a = AMP(s, k), b = AMP(s, k1);
    AMP(s, k) = cadd(cmul(m00, a), cmul(m01, b));
    AMP(s, k1) = cadd(cmul(m10, a), cmul(m11, b));
  }
}

static void apply_cx(double* s, size_t dim, int c, int t) {
  const size_t cm = (size_t)1 << c, tm = (size_t)1 << t;
  for (size_t k = 0; k < dim; ++k) {
    if (!(k & cm) || (k & tm)) continue;
    const cx tmp = AMP(s, k);
    AMP(s, k) = AMP(s, k | tm);
    AMP(s, k | tm) = tmp;
  }
}

static void apply_cy(double* s, size_t dim, int c, int t) {
  const size_t cm = (size_t)1 << c, tm = (size_t)1 << t;
  for (size_t k = 0; k < dim; ++k) {
    if (!(k & cm) || (k & tm)) continue;
    const size_t k1 = k | tm;
    const cx a = AMP(s, k), b = AMP(s, k1);
    AMP(s, k) = cmul(C(0.0, -1.0), b);
    AMP(s, k1) = cmul(C(0.0, 1.0), a);
  }
}

static void apply_ch(double* s, size_t dim, int c, int t) {
  const size_t cm = (size_t)1 << c, tm = (size_t)1 << t;
  const double r = 1.0 / sqrt(2.0);
  for (size_t k = 0; k < dim; ++k) {
    if (!(k & cm) || (k & tm)) continue;
    const size_t k1 = k | tm;
    const cx a = AMP(s, k), b = AMP(s, k1);
    AMP(s, k) = cscale(cadd(a, b), r);
    AMP(s, k1) = cscale(csub(a, b), r);
  }
}

static void apply_controlled_single(double* s, size_t dim, int c, int t, cx m00,
                                    cx m01, cx m10, cx m11) {
  const size_t cm = (size_t)1 << c, tm = (size_t)1 << t;
  for (size_t k = 0; k < dim; ++k) {
    if (!(k & cm) || (k & tm)) continue;
    const size_t k1 = k | tm;
    const cx a = AMP(s, k), b = AMP(s, k1);
    AMP(s, k) = cadd(cmul(m00, a), cmul(m01, b));
    AMP(s, k1) = cadd(cmul(m10, a), cmul(m11, b));
  }
}

static void apply_swap(double* s, size_t dim, int qa, int qb) {
  const size_t ma = (size_t)1 << qa, mb = (size_t)1 << qb;
  for (size_t k = 0; k < dim; ++k) {
    if ((k & ma) && !(k & mb)) {
      const size_t o = (k ^ ma) | mb;
      const cx tmp = AMP(s, k);
      AMP(s, k) = AMP(s, o);
      AMP(s, o) = tmp;
    }
  }
}

static void apply_ccx(double* s, size_t dim, int c1, int c2, int t) {
  const size_t m1 = (size_t)1 << c1, m2 = (size_t)1 << c2, tm = (size_t)1 << t;
  for (size_t k = 0; k < dim; ++k) {
    if (!(k & m1) || !(k & m2)) continue;
    if (k & tm) continue;
    const cx tmp = AMP(s, k);
    AMP(s, k) = AMP(s, k | tm);
    AMP(s, k | tm) = tmp;
  }
}

static void apply_cswap(double* s, size_t dim, int c, int a, int b) {
  const size_t cm = (size_t)1 << c, ma = (size_t)1 << a, mb = (size_t)1 << b;
  for (size_t k = 0; k < dim; ++k) {
    if (!(k & cm)) continue;
    if ((k & ma) && !(k & mb)) {
      const size_t o = (k ^ ma) | mb;
      const cx tmp = AMP(s, k);
      AMP(s, k) = AMP(s, o);
      AMP(s, o) = tmp;
    }
  }
}

static void apply_cphase(double* s, size_t dim, int qa, int qb, cx ph) {
  const size_t ma = (size_t)1 << qa, mb = (size_t)1 << qb;
  for (size_t k = 0; k < dim; ++k) {
    if ((k & ma) && (k & mb)) AMP(s, k) = cmul(AMP(s, k), ph);
  }
}

/* The 2x2 each 1-qubit gate hands to apply_single (simulator.cpp:38-97);
 * also used for the controlled rotations (:168-200). */
static int single_matrix(int type, const double* p, cx m[4]) {
  const double r = 1.0 / sqrt(2.0);
  double c, sn;
  switch (type) {
    case KO_H: m[0] = C(r, 0); m[1] = C(r, 0); m[2] = C(r, 0); m[3] = C(-r, 0); return 0;
    case KO_X: m[0] = C(0, 0); m[1] = C(1, 0); m[2] = C(1, 0); m[3] = C(0, 0); return 0;
    case KO_Y: m[0] = C(0, 0); m[1] = C(0, -1); m[2] = C(0, 1); m[3] = C(0, 0); return 0;
    case KO_Z: m[0] = C(1, 0); m[1] = C(0, 0); m[2] = C(0, 0); m[3] = C(-1, 0); return 0;
    case KO_S: m[0] = C(1, 0); m[1] = C(0, 0); m[2] = C(0, 0); m[3] = C(0, 1); return 0;
    case KO_SDG: m[0] = C(1, 0); m[1] = C(0, 0); m[2] = C(0, 0); m[3] = C(0, -1); return 0;
    case KO_T: m[0] = C(1, 0); m[1] = C(0, 0); m[2] = C(0, 0); m[3] = C(r, r); return 0;
    case KO_TDG: m[0] = C(1, 0); m[1] = C(0, 0); m[2] = C(0, 0); m[3] = C(r, -r); return 0;
    case KO_RX: case KO_CRX:
      c = cos(p[0] / 2.0); sn = sin(p[0] / 2.0);
      m[0] = C(c, 0); m[1] = C(0, -sn); m[2] = C(0, -sn); m[3] = C(c, 0); return 0;
    case KO_RY: case KO_CRY:
      c = cos(p[0] / 2.0); sn = sin(p[0] / 2.0);
      m[0] = C(c, 0); m[1] = C(-sn, 0); m[2] = C(sn, 0); m[3] = C(c, 0); return 0;
    case KO_RZ: case KO_CRZ:
      c = cos(p[0] / 2.0); sn = sin(p[0] / 2.0);
      m[0] = C(c, -sn); m[1] = C(0, 0); m[2] = C(0, 0); m[3] = C(c, sn); return 0;
    case KO_U: case KO_CU:
      c = cos(p[0] / 2.0); sn = sin(p[0] / 2.0);
      m[0] = C(c, 0.0);
      m[1] = cneg(cpolar(sn, p[2]));
      m[2] = cpolar(sn, p[1]);
      m[3] = cpolar(c, p[1] + p[2]);
      return 0;
    default:
      return -1;
  }
}

static int is_unitary(int type) {
  return type >= KO_H && type <= KO_CSWAP;
}

static int gate_arity(int type) {
  if (type <= KO_U) return 1;
  if (type <= KO_SWAP) return 2;
  if (type <= KO_CSWAP) return 3;
  return -1;
}

/* apply_gate_on (simulator.cpp:259-338). */
static void apply_gate_on(double* s, size_t dim, int type, const double* p,
                          const int* on) {
  cx m[4];
  switch (type) {
    case KO_H: case KO_X: case KO_Y: case KO_Z: case KO_S: case KO_SDG:
    case KO_T: case KO_TDG: case KO_RX: case KO_RY: case KO_RZ: case KO_U:
      single_matrix(type, p, m);
      apply_single(s, dim, on[0], m[0], m[1], m[2], m[3]);
      break;
    case KO_CH: apply_ch(s, dim, on[0], on[1]); break;
    case KO_CX: apply_cx(s, dim, on[0], on[1]); break;
    case KO_CY: apply_cy(s, dim, on[0], on[1]); break;
    case KO_CZ: apply_cphase(s, dim, on[0], on[1], C(-1.0, 0.0)); break;
    case KO_CRX: case KO_CRY: case KO_CRZ: case KO_CU:
      single_matrix(type, p, m);
      apply_controlled_single(s, dim, on[0], on[1], m[0], m[1], m[2], m[3]);
      break;
    case KO_CP: apply_cphase(s, dim, on[0], on[1], C(cos(p[0]), sin(p[0]))); break;
    case KO_SWAP: apply_swap(s, dim, on[0], on[1]); break;
    case KO_CCX: apply_ccx(s, dim, on[0], on[1], on[2]); break;
    case KO_CSWAP: apply_cswap(s, dim, on[0], on[1], on[2]); break;
    default: break;
  }
}

int ko_gate_matrix(const ko_op* op, double* m4) {
  cx m[4];
  if (gate_arity(op->type) != 1) return -1;
  if (single_matrix(op->type, op->p, m) != 0) return -1;
  memcpy(m4, m, sizeof m);
  return 0;
}

/* apply_matrix (simulator.cpp:357-393). */
void ko_apply_matrix(int n, double* s, const int* qubits, int m,
                     const double* matd) {
  const size_t dim = (size_t)1 << m;
  const size_t total = (size_t)1 << n;
  const cx* mat = (const cx*)matd;
  int sorted[8];
  size_t offset[64];
  cx in[64], out[64];
  for (int i = 0; i < m; ++i) sorted[i] = qubits[i];
  for (int i = 1; i < m; ++i)
    for (int j = i; j > 0 && sorted[j - 1] > sorted[j]; --j) {
      const int t = sorted[j];
      sorted[j] = sorted[j - 1];
      sorted[j - 1] = t;
    }
  for (size_t i = 0; i < dim; ++i) {
    offset[i] = 0;
    for (int b = 0; b < m; ++b)
      if (i & ((size_t)1 << b)) offset[i] |= (size_t)1 << qubits[b];
  }
  for (size_t o = 0; o < (total >> m); ++o) {
    size_t base = o;
    for (int j = 0; j < m; ++j) {
      const int q = sorted[j];
      base = ((base >> q) << (q + 1)) | (base & (((size_t)1 << q) - 1));
    }
    for (size_t i = 0; i < dim; ++i) in[i] = AMP(s, base | offset[i]);
    for (size_t r = 0; r < dim; ++r) {
      cx acc = C(0.0, 0.0);
      for (size_t c = 0; c < dim; ++c) acc = cadd(acc, cmul(mat[r * dim + c], in[c]));
      out[r] = acc;
    }
    for (size_t i = 0; i < dim; ++i) AMP(s, base | offset[i]) = out[i];
  }
}

/* ---------------------------------------------------------------------------
 * Fuser (simulator.cpp:400-477): a gate joins the open block only if its
 * qubits are a subset of the block's qubits, which the block's first gate
 * fixes; a 1-gate block runs its own loop, a 1-qubit block runs as one 2x2,
 * a wider block as one apply_matrix. */

typedef struct {
  const ko_op** g;
  int (*on)[3];
  int count;
  int qubits[3];
  int nq;
} fuser_t;

static void block_matrix_of(const ko_op* const* gates, int (*on)[3], int count,
                            const int* qubits, int nq, cx* mat) {
  const size_t dim = (size_t)1 << nq;
  double e[2 * 64];
  for (size_t col = 0; col < dim; ++col) {
    memset(e, 0, sizeof(double) * 2 * dim);
    e[2 * col] = 1.0;
    for (int g = 0; g < count; ++g) {
      int local[3];
      const int a = gate_arity(gates[g]->type);
      for (int i = 0; i < a; ++i) {
        local[i] = 0;
        for (int j = 0; j < nq; ++j)
          if (qubits[j] == on[g][i]) local[i] = j;
      }
      apply_gate_on(e, dim, gates[g]->type, gates[g]->p, local);
    }
    for (size_t row = 0; row < dim; ++row) mat[row * dim + col] = AMP(e, row);
  }
}

static void fuser_flush(fuser_t* f, double* s, int n) {
  const size_t dim = (size_t)1 << n;
  if (f->count == 0) return;
  if (f->count == 1) {
    apply_gate_on(s, dim, f->g[0]->type, f->g[0]->p, f->on[0]);
  } else {
    cx mat[64];
    block_matrix_of(f->g, f->on, f->count, f->qubits, f->nq, mat);
    if (f->nq == 1)
      apply_single(s, dim, f->qubits[0], mat[0], mat[1], mat[2], mat[3]);
    else
      ko_apply_matrix(n, s, f->qubits, f->nq, (const double*)mat);
  }
  f->count = 0;
  f->nq = 0;
}

static int is_subset(const int* a, int na, const int* b, int nb) {
  for (int i = 0; i < na; ++i) {
    int found = 0;
    for (int j = 0; j < nb; ++j)
      if (a[i] == b[j]) found = 1;
    if (!found) return 0;
  }
  return 1;
}

void ko_ground_state(int n, double* amps) {
  memset(amps, 0, sizeof(double) * 2 * ((size_t)1 << n));
  amps[0] = 1.0;
}

static int validate(int n, const ko_op* op) {
  if (op->type < 0 || op->type > KO_PROBE) return -1;
  if (!is_unitary(op->type)) return 0;
  const int a = gate_arity(op->type);
  for (int i = 0; i < a; ++i) {
    if (op->q[i] < 0 || op->q[i] >= n) return -1;
    for (int j = 0; j < i; ++j)
      if (op->q[i] == op->q[j]) return -1;
  }
  return 0;
}

int ko_apply(int n, double* s, const ko_op* ops, size_t nops, int fuse_mode) {
  const size_t dim = (size_t)1 << n;
  fuser_t* f = (fuser_t*)calloc(1, sizeof(fuser_t));
  if (!f) return -1;
  f->g = (const ko_op**)malloc(sizeof(ko_op*) * (nops ? nops : 1));
  f->on = (int(*)[3])malloc(sizeof(int[3]) * (nops ? nops : 1));
  if (!f->g || !f->on) {
    free(f->g);
    free(f->on);
    free(f);
    return -1;
  }
  for (size_t i = 0; i < nops; ++i) {
    const ko_op* op = &ops[i];
    if (validate(n, op) != 0) {
      free(f->g);
      free(f->on);
      free(f);
      return -1;
    }
    if (!is_unitary(op->type)) {
      fuser_flush(f, s, n); /* structural ops are fusion barriers */
      continue;
    }
    const int a = gate_arity(op->type);
    if (fuse_mode == KO_FUSE_NONE) {
      apply_gate_on(s, dim, op->type, op->p, op->q);
      continue;
    }
    if (f->count > 0 && !is_subset(op->q, a, f->qubits, f->nq))
      fuser_flush(f, s, n);
    if (f->count == 0) {
      f->nq = a;
      for (int j = 0; j < a; ++j) f->qubits[j] = op->q[j];
    }
    f->g[f->count] = op;
    for (int j = 0; j < a; ++j) f->on[f->count][j] = op->q[j];
    f->count++;
  }
  fuser_flush(f, s, n);
  free(f->g);
  free(f->on);
  free(f);
  return 0;
}

int ko_run(int n, const ko_op* ops, size_t nops, int fuse_mode, double* amps) {
  ko_ground_state(n, amps);
  return ko_apply(n, amps, ops, nops, fuse_mode);
}

int ko_block_matrix(const ko_op* ops, size_t nops, const int* qubits, int k,
                    double* mat) {
  const ko_op** g = (const ko_op**)malloc(sizeof(ko_op*) * (nops ? nops : 1));
  int(*on)[3] = (int(*)[3])malloc(sizeof(int[3]) * (nops ? nops : 1));
  int count = 0;
  if (!g || !on || k < 1 || k > 6) {
    free(g);
    free(on);
    return -1;
  }
  for (size_t i = 0; i < nops; ++i) {
    if (!is_unitary(ops[i].type)) continue;
    const int a = gate_arity(ops[i].type);
    if (!is_subset(ops[i].q, a, qubits, k)) {
      free(g);
      free(on);
      return -1;
    }
    g[count] = &ops[i];
    for (int j = 0; j < a; ++j) on[count][j] = ops[i].q[j];
    count++;
  }
  block_matrix_of(g, on, count, qubits, k, (cx*)mat);
  free(g);
  free(on);
  return 0;
}

/* ---------------------------------------------------------------------------
 * Pauli expectation (observable.cpp:18-83). */

static int pauli_masks(int n, const char* pauli, size_t* flip, size_t* sign,
                       cx* phase) {
  const size_t len = strlen(pauli);
  int num_y = 0;
  *flip = 0;
  *sign = 0;
  if (len != (size_t)n) return -2;
  for (int i = 0; i < n; ++i) {
    char p = pauli[n - 1 - i]; /* rightmost character is qubit 0 */
    if (p >= 'a' && p <= 'z') p = (char)(p - ('a' - 'A'));
    const size_t bit = (size_t)1 << i;
    switch (p) {
      case 'I': break;
      case 'X': *flip |= bit; break;
      case 'Y': *flip |= bit; *sign |= bit; ++num_y; break;
      case 'Z': *sign |= bit; break;
      default: return -3;
    }
  }
  switch (num_y % 4) {
    case 1: *phase = C(0.0, 1.0); break;
    case 2: *phase = C(-1.0, 0.0); break;
    case 3: *phase = C(0.0, -1.0); break;
    default: *phase = C(1.0, 0.0); break;
  }
  return 0;
}

double ko_expval(int n, const double* s, const char* pauli, int* err) {
  size_t flip, sign;
  cx phase;
  const size_t dim = (size_t)1 << n;
  const int rc = pauli_masks(n, pauli, &flip, &sign, &phase);
  if (err) *err = rc;
  if (rc != 0) return 0.0;
  cx sum = C(0.0, 0.0);
  for (size_t x = 0; x < dim; ++x) {
    const cx c = (__builtin_popcountll(x & sign) % 2 == 0) ? phase : cneg(phase);
    sum = cadd(sum, cmul(cmul(c, AMP(s, x)), cconj(AMP(s, x ^ flip))));
  }
  return sum.re;
}

double ko_expval_sum(int n, const double* s, const double* coeffs,
                     const char* const* paulis, size_t nterms, int* err) {
  double total = 0.0;
  if (err) *err = 0;
  for (size_t t = 0; t < nterms; ++t) {
    int e = 0;
    const double v = ko_expval(n, s, paulis[t], &e);
    if (e != 0) {
      if (err) *err = e;
      return 0.0;
    }
    total += coeffs[t] * v;
  }
  return total;
}

/* ---------------------------------------------------------------------------
 * Born-rule draws (measurement.cpp:12-21). */

static inline double norm_at(const double* s, const float* s32, size_t i) {
  if (s) {
    const double x = s[2 * i], y = s[2 * i + 1];
    return x * x + y * y;
  }
  const double x = (double)s32[2 * i], y = (double)s32[2 * i + 1];
  return x * x + y * y;
}

uint64_t ko_measure_sequential(int n, const double* s, double u) {
  const size_t dim = (size_t)1 << n;
  double cum = 0.0;
  for (size_t i = 0; i < dim; ++i) {
    cum += norm_at(s, NULL, i);
    if (u < cum) return i;
  }
  return dim - 1;
}

typedef struct {
  double u;
  size_t idx;
} ukey;

static int cmp_ukey(const void* a, const void* b) {
  const double x = ((const ukey*)a)->u, y = ((const ukey*)b)->u;
  return (x > y) - (x < y);
}

static void measure_sequential_many_any(int n, const double* s, const float* s32, const double* u,
                                        size_t count, uint64_t* out);

void ko_measure_sequential_many(int n, const double* s, const double* u,
                                size_t count, uint64_t* out) {
  measure_sequential_many_any(n, s, NULL, u, count, out);
}

void ko_measure_sequential_many32(int n, const float* s32, const double* u,
                                  size_t count, uint64_t* out) {
  measure_sequential_many_any(n, NULL, s32, u, count, out);
}

static void measure_sequential_many_any(int n, const double* s, const float* s32, const double* u,
                                        size_t count, uint64_t* out) {
  const size_t dim = (size_t)1 << n;
  ukey* keys = (ukey*)malloc(sizeof(ukey) * (count ? count : 1));
  for (size_t j = 0; j < count; ++j) {
    keys[j].u = u[j];
    keys[j].idx = j;
  }
  qsort(keys, count, sizeof(ukey), cmp_ukey);
  double cum = 0.0;
  size_t j = 0;
  for (size_t i = 0; i < dim && j < count; ++i) {
    cum += norm_at(s, s32, i);
    while (j < count && keys[j].u < cum) out[keys[j++].idx] = i;
  }
  while (j < count) out[keys[j++].idx] = dim - 1;
  free(keys);
}

/* MT19937 (Matsumoto & Nishimura 1998) as std::mt19937, and libstdc++'s
 * generate_canonical<double, 53>: two words w0 + w1 * 2^32, divided by 2^64,
 * clamped below 1. */
void ko_uniforms_mt19937(uint32_t seed, size_t count, double* out) {
  uint32_t mt[624];
  int idx = 624;
  mt[0] = seed;
  for (int i = 1; i < 624; ++i)
    mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (uint32_t)i;
  for (size_t d = 0; d < count; ++d) {
    double sum = 0.0, scale = 1.0;
    for (int w = 0; w < 2; ++w) {
      if (idx >= 624) {
        for (int i = 0; i < 624; ++i) {
          const uint32_t y = (mt[i] & 0x80000000u) | (mt[(i + 1) % 624] & 0x7fffffffu);
          mt[i] = mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        idx = 0;
      }
      uint32_t y = mt[idx++];
      y ^= y >> 11;
      y ^= (y << 7) & 0x9d2c5680u;
      y ^= (y << 15) & 0xefc60000u;
      y ^= y >> 18;
      sum += (double)y * scale;
      scale *= 4294967296.0;
    }
    double r = sum / scale;
    if (r >= 1.0) r = nextafter(1.0, 0.0);
    out[d] = r;
  }
}

/* Fixed-tree sampler (the backend's documented summation order). */
void ko_sample_tree(int n, const double* s, const float* s32, const double* u,
                    size_t count, uint64_t* out) {
  const size_t N = (size_t)1 << n;
  const size_t S = KO_SEG;
  /* level sizes */
  size_t sizes[64];
  double* V[64]; /* V[l] for l >= 1: segment totals */
  double* F[64]; /* inclusive carries at level l >= 1 */
  int L = 0;
  sizes[0] = N;
  while (sizes[L] > S) {
    sizes[L + 1] = (sizes[L] + S - 1) / S;
    ++L;
  }
  for (int l = 1; l <= L; ++l) {
    V[l] = (double*)malloc(sizeof(double) * sizes[l]);
    F[l] = (double*)malloc(sizeof(double) * sizes[l]);
    for (size_t j = 0; j < sizes[l]; ++j) {
      double acc = 0.0;
      const size_t lo = j * S, hi = (lo + S < sizes[l - 1]) ? lo + S : sizes[l - 1];
      for (size_t i = lo; i < hi; ++i)
        acc += (l == 1) ? norm_at(s, s32, i) : V[l - 1][i];
      V[l][j] = acc;
    }
  }
  /* top-down inclusive carries */
  if (L >= 1) {
    double c = 0.0;
    for (size_t j = 0; j < sizes[L]; ++j) {
      c += V[L][j];
      F[L][j] = c;
    }
    for (int l = L - 1; l >= 1; --l) {
      for (size_t jp = 0; jp < sizes[l + 1]; ++jp) {
        double c2 = (jp == 0) ? 0.0 : F[l + 1][jp - 1];
        const size_t lo = jp * S, hi = (lo + S < sizes[l]) ? lo + S : sizes[l];
        for (size_t j = lo; j < hi; ++j) {
          c2 += V[l][j];
          F[l][j] = c2;
        }
      }
    }
  }
  for (size_t d = 0; d < count; ++d) {
    const double x = u[d];
    double carry = 0.0;
    size_t lo = 0, hi = sizes[L];
    for (int l = L; l >= 1; --l) {
      size_t pick = hi - 1;
      for (size_t j = lo; j < hi; ++j)
        if (x < F[l][j]) {
          pick = j;
          break;
        }
      carry = (pick == lo) ? carry : F[l][pick - 1];
      lo = pick * S;
      hi = (lo + S < sizes[l - 1]) ? lo + S : sizes[l - 1];
    }
    size_t pick = hi - 1;
    double c = carry;
    for (size_t i = lo; i < hi; ++i) {
      c += norm_at(s, s32, i);
      if (x < c) {
        pick = i;
        break;
      }
    }
    out[d] = pick;
  }
  for (int l = 1; l <= L; ++l) {
    free(V[l]);
    free(F[l]);
  }
}

/* ---------------------------------------------------------------------------
 * Adjoint reference: straightforward FP64 reverse sweep.  The derivative of
 * each parameterised gate is applied explicitly as a (non-unitary) matrix;
 * <lambda| dU psi_prev> is summed over the whole vector. */

static void apply_ctrl2x2(double* s, size_t dim, size_t cmask, int t,
                          const cx m[4]) {
  const size_t tm = (size_t)1 << t;
  for (size_t k = 0; k < dim; ++k) {
    if ((k & cmask) != cmask || (k & tm)) continue;
    const size_t k1 = k | tm;
    const cx a = AMP(s, k), b = AMP(s, k1);
    AMP(s, k) = cadd(cmul(m[0], a), cmul(m[1], b));
    AMP(s, k1) = cadd(cmul(m[2], a), cmul(m[3], b));
  }
}

static void dagger2(const cx m[4], cx d[4]) {
  d[0] = cconj(m[0]);
  d[1] = cconj(m[2]);
  d[2] = cconj(m[1]);
  d[3] = cconj(m[3]);
}

/* Apply op (or its inverse) as a controlled 2x2 / permutation. */
static void apply_generic(double* s, size_t dim, const ko_op* op, double th,
                          int inverse) {
  double p[3] = {op->p[0], op->p[1], op->p[2]};
  cx m[4], d[4];
  p[0] = th;
  const int t = op->type;
  if (t == KO_SWAP || t == KO_CSWAP || t == KO_CX || t == KO_CCX) {
    apply_gate_on(s, dim, t, p, op->q);
    return;
  }
  if (t == KO_CZ || t == KO_CP) {
    cx ph = (t == KO_CZ) ? C(-1.0, 0.0) : C(cos(th), sin(th));
    if (inverse) ph = cconj(ph);
    apply_cphase(s, dim, op->q[0], op->q[1], ph);
    return;
  }
  size_t cmask = 0;
  int tq;
  int base = t;
  if (t == KO_CH) {
    base = KO_H;
  } else if (t == KO_CY) {
    base = KO_Y;
  }
  if (gate_arity(t) == 2) {
    cmask = (size_t)1 << op->q[0];
    tq = op->q[1];
  } else {
    tq = op->q[0];
  }
  single_matrix(base == KO_CRX ? KO_RX : base == KO_CRY ? KO_RY
                : base == KO_CRZ ? KO_RZ : base == KO_CU ? KO_U : base,
                p, m);
  if (inverse) {
    dagger2(m, d);
    apply_ctrl2x2(s, dim, cmask, tq, d);
  } else {
    apply_ctrl2x2(s, dim, cmask, tq, m);
  }
}

/* d/dtheta of the op's matrix applied to s (zero outside the controlled
 * subspace).  Supported: Rx, Ry, Rz, CRx, CRy, CRz, CP, U (theta). */
static int apply_derivative(double* s, size_t dim, const ko_op* op, double th) {
  const double c = cos(th / 2.0), sn = sin(th / 2.0);
  cx m[4];
  size_t cmask = 0;
  int tq = op->q[0];
  switch (op->type) {
    case KO_RX: case KO_CRX:
      m[0] = C(-sn / 2, 0); m[1] = C(0, -c / 2); m[2] = C(0, -c / 2); m[3] = C(-sn / 2, 0);
      break;
    case KO_RY: case KO_CRY:
      m[0] = C(-sn / 2, 0); m[1] = C(-c / 2, 0); m[2] = C(c / 2, 0); m[3] = C(-sn / 2, 0);
      break;
    case KO_RZ: case KO_CRZ:
      m[0] = C(-sn / 2, -c / 2); m[1] = C(0, 0); m[2] = C(0, 0); m[3] = C(-sn / 2, c / 2);
      break;
    case KO_U:
      m[0] = C(-sn / 2, 0.0);
      m[1] = cneg(cpolar(c / 2, op->p[2]));
      m[2] = cpolar(c / 2, op->p[1]);
      m[3] = cpolar(-sn / 2, op->p[1] + op->p[2]);
      break;
    case KO_CP: {
      const size_t ma = (size_t)1 << op->q[0], mb = (size_t)1 << op->q[1];
      const cx d = C(-sin(th), cos(th));
      for (size_t k = 0; k < dim; ++k) {
        if ((k & ma) && (k & mb)) AMP(s, k) = cmul(AMP(s, k), d);
        else AMP(s, k) = C(0.0, 0.0);
      }
      return 0;
    }
    default:
      return -1;
  }
  if (gate_arity(op->type) == 2) {
    cmask = (size_t)1 << op->q[0];
    tq = op->q[1];
  }
  const size_t tm = (size_t)1 << tq;
  for (size_t k = 0; k < dim; ++k) {
    if (k & tm) continue;
    const size_t k1 = k | tm;
    if ((k & cmask) != cmask) {
      AMP(s, k) = C(0.0, 0.0);
      AMP(s, k1) = C(0.0, 0.0);
      continue;
    }
    const cx a = AMP(s, k), b = AMP(s, k1);
    AMP(s, k) = cadd(cmul(m[0], a), cmul(m[1], b));
    AMP(s, k1) = cadd(cmul(m[2], a), cmul(m[3], b));
  }
  return 0;
}

/* lambda = H psi, H = sum_t coeff_t P_t; (P psi)[y] =
 * phase * (-1)^popcount((y^flip)&sign) * psi[y^flip] (from observable.cpp:68-83). */
static int apply_hamiltonian(int n, const double* psi, const double* coeffs,
                             const char* const* paulis, size_t nterms,
                             double* out) {
  const size_t dim = (size_t)1 << n;
  memset(out, 0, sizeof(double) * 2 * dim);
  for (size_t t = 0; t < nterms; ++t) {
    size_t flip, sign;
    cx phase;
    const int rc = pauli_masks(n, paulis[t], &flip, &sign, &phase);
    if (rc != 0) return rc;
    for (size_t y = 0; y < dim; ++y) {
      const size_t x = y ^ flip;
      cx c = (__builtin_popcountll(x & sign) % 2 == 0) ? phase : cneg(phase);
      c = cscale(c, coeffs[t]);
      AMP(out, y) = cadd(AMP(out, y), cmul(c, AMP(psi, x)));
    }
  }
  return 0;
}

int ko_adjoint(int n, const ko_op* ops, size_t nops, const int* param_index,
               const double* params, size_t nparams, const double* coeffs,
               const char* const* paulis, size_t nterms, double* value,
               double* grad) {
  const size_t dim = (size_t)1 << n;
  double* psi = (double*)malloc(sizeof(double) * 2 * dim);
  double* lam = (double*)malloc(sizeof(double) * 2 * dim);
  double* phi = (double*)malloc(sizeof(double) * 2 * dim);
  if (!psi || !lam || !phi) return -1;
  for (size_t i = 0; i < nparams; ++i) grad[i] = 0.0;
  ko_ground_state(n, psi);
  for (size_t i = 0; i < nops; ++i) {
    if (!is_unitary(ops[i].type)) continue;
    const double th = (param_index && param_index[i] >= 0) ? params[param_index[i]] : ops[i].p[0];
    apply_generic(psi, dim, &ops[i], th, 0);
  }
  int rc = apply_hamiltonian(n, psi, coeffs, paulis, nterms, lam);
  if (rc != 0) {
    free(psi); free(lam); free(phi);
    return rc;
  }
  double v = 0.0;
  for (size_t x = 0; x < dim; ++x) v += psi[2 * x] * lam[2 * x] + psi[2 * x + 1] * lam[2 * x + 1];
  *value = v;
  for (size_t ii = nops; ii-- > 0;) {
    const ko_op* op = &ops[ii];
    if (!is_unitary(op->type)) continue;
    const double th = (param_index && param_index[ii] >= 0) ? params[param_index[ii]] : op->p[0];
    apply_generic(psi, dim, op, th, 1); /* psi <- psi_{i-1} */
    if (param_index && param_index[ii] >= 0) {
      memcpy(phi, psi, sizeof(double) * 2 * dim);
      if (apply_derivative(phi, dim, op, th) != 0) {
        free(psi); free(lam); free(phi);
        return -1;
      }
      double acc = 0.0;
      for (size_t x = 0; x < dim; ++x)
        acc += lam[2 * x] * phi[2 * x] + lam[2 * x + 1] * phi[2 * x + 1];
      grad[param_index[ii]] += 2.0 * acc;
    }
    apply_generic(lam, dim, op, th, 1);
  }
  free(psi);
  free(lam);
  free(phi);
  return 0;
}

/* ---------------------------------------------------------------------------
 * MLP reference: y = w3 . relu(W2 relu(W1 x + b1) + b2) + b3, row-major
 * weights W1[128][48], W2[128][128], w3[128]. */

#define MI 48
#define MH 128

void ko_mlp_forward(const float* w1, const float* b1, const float* w2,
                    const float* b2, const float* w3, const float* b3,
                    const float* x, int batch, double* out) {
  double h1[MH], h2[MH];
  for (int b = 0; b < batch; ++b) {
    for (int i = 0; i < MH; ++i) {
      double a = b1[i];
      for (int k = 0; k < MI; ++k) a += (double)w1[i * MI + k] * x[b * MI + k];
      h1[i] = a > 0 ? a : 0;
    }
    for (int i = 0; i < MH; ++i) {
      double a = b2[i];
      for (int k = 0; k < MH; ++k) a += (double)w2[i * MH + k] * h1[k];
      h2[i] = a > 0 ? a : 0;
    }
    double o = b3[0];
    for (int k = 0; k < MH; ++k) o += (double)w3[k] * h2[k];
    out[b] = o;
  }
}

double ko_mlp_backward(const float* w1, const float* b1, const float* w2,
                       const float* b2, const float* w3, const float* b3,
                       const float* x, const float* y, int batch, double* gw1,
                       double* gb1, double* gw2, double* gb2, double* gw3,
                       double* gb3) {
  double h1[MH], h2[MH], z1[MH], z2[MH], d2[MH], d1[MH];
  double loss = 0.0;
  memset(gw1, 0, sizeof(double) * MH * MI);
  memset(gb1, 0, sizeof(double) * MH);
  memset(gw2, 0, sizeof(double) * MH * MH);
  memset(gb2, 0, sizeof(double) * MH);
  memset(gw3, 0, sizeof(double) * MH);
  gb3[0] = 0.0;
  for (int b = 0; b < batch; ++b) {
    for (int i = 0; i < MH; ++i) {
      double a = b1[i];
      for (int k = 0; k < MI; ++k) a += (double)w1[i * MI + k] * x[b * MI + k];
      z1[i] = a;
      h1[i] = a > 0 ? a : 0;
    }
    for (int i = 0; i < MH; ++i) {
      double a = b2[i];
      for (int k = 0; k < MH; ++k) a += (double)w2[i * MH + k] * h1[k];
      z2[i] = a;
      h2[i] = a > 0 ? a : 0;
    }
    double o = b3[0];
    for (int k = 0; k < MH; ++k) o += (double)w3[k] * h2[k];
    const double e = o - y[b];
    loss += e * e / batch;
    const double go = 2.0 * e / batch;
    gb3[0] += go;
    for (int k = 0; k < MH; ++k) {
      gw3[k] += go * h2[k];
      d2[k] = (z2[k] > 0) ? go * w3[k] : 0.0;
    }
    for (int i = 0; i < MH; ++i) {
      gb2[i] += d2[i];
      for (int k = 0; k < MH; ++k) gw2[i * MH + k] += d2[i] * h1[k];
    }
    for (int k = 0; k < MH; ++k) {
      double a = 0.0;
      for (int i = 0; i < MH; ++i) a += d2[i] * w2[i * MH + k];
      d1[k] = (z1[k] > 0) ? a : 0.0;
    }
    for (int i = 0; i < MH; ++i) {
      gb1[i] += d1[i];
      for (int k = 0; k < MI; ++k) gw1[i * MI + k] += d1[i] * x[b * MI + k];
    }
  }
  return loss;
}
