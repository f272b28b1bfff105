/*
 * ketsv_oracle.h -- CPU oracle for the ket state-vector path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (ket's src/simulator.cpp, src/observable.cpp and
 * src/measurement.cpp) used as the checker for the CUDA backend.  Only the
 * test suite, the smoke check and the CPU-baseline leg of the benchmark load
 * it; the product library never links or calls it.
 *
 * Amplitudes are complex128 stored interleaved (re, im) in a double array of
 * length 2 * 2^n, index bit q = qubit q (little-endian), as in ket's State
 * (include/ket/state.hpp:12-34).
 */
#ifndef KETSV_ORACLE_H
#define KETSV_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Gate codes: identical numbering to ket::GateType (include/ket/gate.hpp:16-29). */
enum {
  KO_H = 0, KO_X, KO_Y, KO_Z, KO_S, KO_SDG, KO_T, KO_TDG, KO_RX, KO_RY, KO_RZ,
  KO_U, KO_CH, KO_CX, KO_CY, KO_CZ, KO_CRX, KO_CRY, KO_CRZ, KO_CU, KO_CP,
  KO_SWAP, KO_CCX, KO_CSWAP, KO_MEASURE, KO_BARRIER, KO_COMPOSITE, KO_PROBE
};

/* One flat circuit operation; same 48-byte layout as ketgpu_op in
 * include/ket_b200.h.  For MEASURE, q[1] holds the classical bit. */
typedef struct ko_op {
  int32_t type;
  int32_t nq;
  int32_t q[3];
  int32_t aux;
  double p[3];
} ko_op;

/* Fusion modes of ko_apply. */
enum {
  KO_FUSE_NONE = 0,      /* every gate through its own per-gate loop */
  KO_FUSE_REFERENCE = 1  /* ket's Fuser (simulator.cpp:400-477), as ket::run does */
};

/* |0...0> into amps (2 * 2^n doubles). */
void ko_ground_state(int n, double* amps);

/* Apply ops to amps in place.  Returns 0, or -1 on a malformed op. */
int ko_apply(int n, double* amps, const ko_op* ops, size_t nops, int fuse_mode);

/* ket::run restated: ground state, then ko_apply with the reference fuser. */
int ko_run(int n, const ko_op* ops, size_t nops, int fuse_mode, double* amps);

/* Dense m-qubit apply (simulator.cpp:357-393): mat is row-major 2^m x 2^m
 * complex (interleaved), bit b of the matrix index <-> qubits[b]. */
void ko_apply_matrix(int n, double* amps, const int* qubits, int m,
                     const double* mat);

/* 2x2 block matrix of a single gate (row-major, interleaved) as the
 * reference's per-gate loops apply it; returns 0 for 1-qubit unitary gates. */
int ko_gate_matrix(const ko_op* op, double* m4);

/* The 2^k x 2^k matrix of a gate sequence over local qubits `qubits` (bit b
 * <-> qubits[b]), built column by column as Fuser::block_matrix does
 * (simulator.cpp:448-465).  Returns 0 or -1. */
int ko_block_matrix(const ko_op* ops, size_t nops, const int* qubits, int k,
                    double* mat);

/* Pauli-string expectation (observable.cpp:18-83): err = 0 ok, -1 size not a
 * power of two, -2 length mismatch, -3 bad character. */
double ko_expval(int n, const double* amps, const char* pauli, int* err);

/* Coefficient-weighted sum (observable.cpp:85-91). */
double ko_expval_sum(int n, const double* amps, const double* coeffs,
                     const char* const* paulis, size_t nterms, int* err);

/* ket::measure's sequential CDF scan for one uniform u (measurement.cpp:12-21). */
uint64_t ko_measure_sequential(int n, const double* amps, double u);

/* Same scan for many uniforms, all answered in one ordered pass. */
void ko_measure_sequential_many(int n, const double* amps, const double* u,
                                size_t count, uint64_t* out);

/* The same for a complex64 state (probabilities computed in FP64). */
void ko_measure_sequential_many32(int n, const float* amps32, const double* u,
                                  size_t count, uint64_t* out);

/* std::mt19937{seed} followed by uniform_real_distribution<double>(0,1)
 * draws, restated from the published MT19937 and libstdc++'s
 * generate_canonical<double,53> (two 32-bit words per draw). */
void ko_uniforms_mt19937(uint32_t seed, size_t count, double* out);

/* ---- fixed-tree sampler (the backend's documented CDF) -------------------
 * probabilities p[i] = re*re + im*im in FP64 (no fused multiply-add);
 * level-0 segments of KO_SEG consecutive entries; T_l[j] = sequential sum of
 * segment j of level l-1 starting from 0.0; carries are propagated top-down
 * as sequential folds.  A draw u descends level by level, at each level taking
 * the first child whose running carry exceeds u (the reference's rule,
 * measurement.cpp:15-19, applied to coarser totals), else the last child. */
#define KO_SEG 32
/* Sample `count` uniforms from a complex128 state (amps) or a complex64 state
 * (amps32, used when amps == NULL). */
void ko_sample_tree(int n, const double* amps, const float* amps32,
                    const double* u, size_t count, uint64_t* out);

/* ---- adjoint / gradients (no reference counterpart: restated from the gate
 * algebra of simulator.cpp:73-97 and the Pauli algebra of
 * observable.cpp:68-83) ---------------------------------------------------
 * ops: the circuit; param_index[i] >= 0 marks op i's first angle as the
 * parameter with that index (Rx/Ry/Rz/CRx/CRy/CRz/CP/U theta).  params
 * overrides those angles.  Writes <H> to *value and dH/dparam to grad. */
int ko_adjoint(int n, const ko_op* ops, size_t nops, const int* param_index,
               const double* params, size_t nparams, const double* coeffs,
               const char* const* paulis, size_t nterms, double* value,
               double* grad);

/* ---- MLP cost model reference (48 -> 128 -> 128 -> 1, ReLU) ------------- */
/* Weights are given as float (already rounded to bf16 by the caller);
 * computes in double.  x: batch x 48, out: batch. */
void ko_mlp_forward(const float* w1, const float* b1, const float* w2,
                    const float* b2, const float* w3, const float* b3,
                    const float* x, int batch, double* out);
/* Mean-squared-error loss and gradients w.r.t. every weight (double). */
double ko_mlp_backward(const float* w1, const float* b1, const float* w2,
                       const float* b2, const float* w3, const float* b3,
                       const float* x, const float* y, int batch, double* gw1,
                       double* gb1, double* gw2, double* gb2, double* gw3,
                       double* gb3);

#ifdef __cplusplus
}
#endif

#endif
