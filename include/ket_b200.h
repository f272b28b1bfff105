/*
 * ket_b200.h -- C ABI of the B200 state-vector backend for ket.
 *
 * The library (ket_b200/libket_b200.so) holds every CUDA kernel of the
 * backend.  Its entry points take plain pointers and sizes only, so ket's
 * C++ layer (or any FFI) can bind them without CUDA or torch headers.  Each
 * declaration names the reference interface it replaces, as
 * file:line within the ket sources.
 *
 * Conventions
 *   - Every function returns KETGPU_OK (0) or a negative KETGPU_ERR_* code;
 *     ketgpu_last_error() gives the calling thread's last message.  The
 *     codes map onto the exceptions ket throws: OUT_OF_RANGE ->
 *     std::out_of_range, INVALID -> std::invalid_argument, LOGIC ->
 *     std::logic_error, anything else -> std::runtime_error.
 *   - Host buffers of amplitudes are complex128 interleaved (re, im), index
 *     bit q = qubit q (little-endian), exactly ket::State's layout
 *     (include/ket/state.hpp:12-34).
 *   - A ketgpu_state lives on the CUDA device that was current when it was
 *     created; calls switch to that device and back.
 *   - Calls that return a result to the host synchronise the state's stream;
 *     ketgpu_plan_execute only enqueues.
 */
#ifndef KET_B200_H
#define KET_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KETGPU_ABI_VERSION 1

#define KETGPU_OK 0
#define KETGPU_ERR_OUT_OF_RANGE (-1)
#define KETGPU_ERR_INVALID (-2)
#define KETGPU_ERR_LOGIC (-3)
#define KETGPU_ERR_CUDA (-4)
#define KETGPU_ERR_OOM (-5)
#define KETGPU_ERR_TIMEOUT (-6)

/* Gate codes: the numbering of ket::GateType (include/ket/gate.hpp:16-29). */
enum ketgpu_gate {
  KETGPU_H = 0, KETGPU_X, KETGPU_Y, KETGPU_Z, KETGPU_S, KETGPU_SDG, KETGPU_T,
  KETGPU_TDG, KETGPU_RX, KETGPU_RY, KETGPU_RZ, KETGPU_U, KETGPU_CH, KETGPU_CX,
  KETGPU_CY, KETGPU_CZ, KETGPU_CRX, KETGPU_CRY, KETGPU_CRZ, KETGPU_CU,
  KETGPU_CP, KETGPU_SWAP, KETGPU_CCX, KETGPU_CSWAP, KETGPU_MEASURE,
  KETGPU_BARRIER, KETGPU_COMPOSITE, KETGPU_PROBE
};

/* One circuit operation, the flattened form of ket::Gate
 * (include/ket/gate.hpp:31-41): qubits in g.qubits order, params in
 * g.params order.  Composite blocks are flattened by the caller (wire
 * remap as in simulator.cpp:504-511).  For MEASURE, q[1] is the classical
 * bit.  48 bytes. */
typedef struct ketgpu_op {
  int32_t type;
  int32_t nq;
  int32_t q[3];
  int32_t aux;
  double p[3];
} ketgpu_op;

enum ketgpu_precision { KETGPU_C64 = 0, KETGPU_C128 = 1 };

enum ketgpu_fusion {
  KETGPU_FUSE_NONE = 0,      /* the plain method: one kernel per gate, except
                                consecutive gates on qubits 0..10 share one
                                pass over chunks staged in shared memory */
  KETGPU_FUSE_REFERENCE = 1, /* ket's own block rule (simulator.cpp:400-477) */
  KETGPU_FUSE_GREEDY = 2,    /* DAG-aware k-qubit blocks, static cost model */
  KETGPU_FUSE_LEARNED = 3    /* k-qubit blocks scored by the MLP cost model */
};

typedef struct ketgpu_options {
  int32_t precision;        /* ketgpu_precision */
  int32_t fusion;           /* ketgpu_fusion */
  int32_t max_block_qubits; /* k <= 6 (fused blocks); 0 = default: 6 for
                               complex64 with tensor_cores, else 5 */
  int32_t tensor_cores;     /* 1: complex64 blocks on tcgen05 (3xFP16); 0: SIMT */
  int32_t renormalize;      /* 0: restore the starting norm after tensor-core
                               blocks (their FP32 accumulation rounds toward
                               zero); -1: never; 1: after every plan */
} ketgpu_options;

typedef struct ketgpu_plan_stats {
  uint64_t n_gates;         /* unitary gates in the circuit */
  uint64_t n_passes;        /* kernels one execution launches */
  uint64_t n_fused;         /* dense k-qubit block passes among them */
  uint64_t n_tensor;        /* of those, on the tensor cores */
  double bytes;             /* algorithmic HBM bytes of one execution */
  double flops;             /* algorithmic flops of the fused blocks */
  double predicted_us;      /* cost-model estimate (learned / greedy) */
} ketgpu_plan_stats;

typedef struct ketgpu_state ketgpu_state;
typedef struct ketgpu_plan ketgpu_plan;
typedef struct ketgpu_mlp ketgpu_mlp;

/* ---- library --------------------------------------------------------- */
const char* ketgpu_last_error(void);
int ketgpu_abi_version(void);
/* Number of launches of this library's kernels since load (all devices). */
uint64_t ketgpu_launch_count(void);

/* ---- state: replaces ket::State storage and ground_state
 *      (include/ket/state.hpp:15-34, src/simulator.cpp:529-533) ---------- */
int ketgpu_state_create(int32_t n_qubits, int32_t precision, ketgpu_state** out);
int ketgpu_state_destroy(ketgpu_state* s);
int ketgpu_state_reset(ketgpu_state* s); /* |0...0> */
int ketgpu_state_info(const ketgpu_state* s, int32_t* n_qubits, int32_t* precision);
/* Device pointer of the amplitudes (float2 or double2 per amplitude).  The
 * call counts as a write (the caller may change amplitudes through the
 * pointer), so the next ketgpu_sample rebuilds the sampling tree; call it
 * again after writing through a pointer obtained earlier. */
void* ketgpu_state_device_ptr(const ketgpu_state* s);
/* Copy amplitudes [first, first+count) to a host complex128 buffer. */
int ketgpu_state_download(const ketgpu_state* s, uint64_t first, uint64_t count,
                          double* out_c128);
/* Copy amplitudes [first, first+count) to a host buffer in the state's own
 * format (complex64 or complex128 interleaved), without conversion. */
int ketgpu_state_download_raw(const ketgpu_state* s, uint64_t first, uint64_t count, void* out);
/* Overwrite amplitudes [first, first+count) from a host complex128 buffer. */
int ketgpu_state_upload(ketgpu_state* s, uint64_t first, uint64_t count,
                        const double* in_c128);
int ketgpu_state_copy(const ketgpu_state* src, ketgpu_state* dst);
int ketgpu_state_synchronize(ketgpu_state* s);

/* ---- circuits: replaces ket::run / apply_circuit / Fuser
 *      (include/ket/simulator.hpp:15, src/simulator.cpp:400-558) --------- */
int ketgpu_plan_create(int32_t n_qubits, const ketgpu_op* ops, uint64_t n_ops,
                       const ketgpu_options* opt, ketgpu_plan** out);
int ketgpu_plan_destroy(ketgpu_plan* p);
int ketgpu_plan_stats_get(const ketgpu_plan* p, ketgpu_plan_stats* out);
/* Enqueue every pass of the plan on the state's stream (no host sync). */
int ketgpu_plan_execute(const ketgpu_plan* p, ketgpu_state* s);
/* Execute and time every pass with CUDA events on the state's stream;
 * pass_ms receives n_passes durations (milliseconds).  Synchronises. */
int ketgpu_plan_execute_timed(const ketgpu_plan* p, ketgpu_state* s, float* pass_ms);
/* Describe pass `index`: kind (0 pair, 1 phase, 2 dense block, 3 norm
 * capture/restore, 4 diagonal run, 5 shared-memory run of low-qubit gates),
 * k (block qubits, the qubits a diagonal run touches, or a shared-memory
 * run's gate count), tensor-core flag and algorithmic HBM bytes. */
int ketgpu_plan_pass_info(const ketgpu_plan* p, uint64_t index, int32_t* kind, int32_t* k,
                          int32_t* tensor, double* bytes);
/* The qubits pass `index` acts on, ascending: a dense block's qubits (matrix
 * bit b <-> qubits[b]), or a pair/phase pass's target and controls.  Writes
 * min(count, capacity) entries; *count receives the full number (0 for norm
 * passes and diagonal runs, which touch every qubit). */
int ketgpu_plan_pass_qubits(const ketgpu_plan* p, uint64_t index, int32_t* qubits,
                            int32_t capacity, int32_t* count);
/* The circuit ops (indices into the plan's op array) that pass `index`
 * applies, in the order it applies them.  The planner may reorder commuting
 * gates (its band orders), so the passes' gate lists, concatenated, are a
 * topological order of the circuit's gates.  Writes min(count, capacity)
 * entries; *count receives the full number (0 for norm passes).  Host only;
 * no counterpart in ket. */
int ketgpu_plan_pass_gates(const ketgpu_plan* p, uint64_t index, int32_t* gates,
                           int32_t capacity, int32_t* count);
/* How tensor-core pass `index` runs: tma_dims = dimensions of the tensor map
 * that fetches each tile with one tiled copy (0: per-thread cp.async), and
 * direct = 1 when the epilogue stores straight from registers (0: staged
 * through shared memory).  Assumes the driver provides cuTensorMapEncodeTiled.
 * KETGPU_ERR_INVALID for a pass that is not a tensor-core block.  Host only;
 * no counterpart in ket. */
int ketgpu_plan_pass_tc_form(const ketgpu_plan* p, uint64_t index, int32_t* tma_dims,
                             int32_t* direct);
/* The FP64 matrix of dense-block pass `index` (2^k x 2^k complex, row-major,
 * interleaved re, im; matrix bit b <-> the pass's qubit b), as the plan
 * built it from the pass's gates.  Writes min(capacity, 2 * 4^k) doubles;
 * *count receives 2 * 4^k.  KETGPU_ERR_INVALID for a pass that is not a
 * dense block.  Host only; no counterpart in ket. */
int ketgpu_plan_pass_matrix(const ketgpu_plan* p, uint64_t index, double* out, uint64_t capacity,
                            uint64_t* count);
/* The tensor-core B operand of a k-qubit block (k = 4, 5 or 6) as plans
 * upload it: the real embedding of `mat` (2^k x 2^k complex, row-major,
 * interleaved re, im) scaled by 2^sb (its largest entry into [2^14, 2^15)),
 * split into fp16 hi = round(x) and lo = round(x - hi), as two K-major
 * 128-byte-swizzled images (hi, then lo, each in whole 128-byte atoms along
 * K), then sb as a 32-bit integer.  Writes min(capacity, size) 32-bit words;
 * *words receives the size.  Host only; no counterpart in ket. */
int ketgpu_tc_image(int32_t k, const double* mat, uint32_t* out, uint64_t capacity, uint64_t* words);
/* The state's CUDA stream (a cudaStream_t), for callers that order their
 * own work or events against the backend's. */
void* ketgpu_state_stream(const ketgpu_state* s);
/* Plan + execute + synchronise. */
int ketgpu_apply(ketgpu_state* s, const ketgpu_op* ops, uint64_t n_ops,
                 const ketgpu_options* opt);
/* ket::run with host buffers: |0...0>, the circuit, then the 2^n amplitudes
 * as complex128 into out_c128 (simulator.hpp:15, simulator.cpp:554-558).
 * The device state is kept after the call and reused by the next call of
 * the same size, precision and device: freeing a 30-qubit state costs
 * 150-700 ms.  A state allocation that would not fit frees it first, and
 * ketgpu_release_cache frees it at once.  Concurrent calls each use their
 * own state. */
int ketgpu_run(int32_t n_qubits, const ketgpu_op* ops, uint64_t n_ops,
               const ketgpu_options* opt, double* out_c128);
/* Host wall time of the phases of the calling thread's last ketgpu_run, in
 * milliseconds: out6 = {plan (validate + fusion + block matrices), state
 * (reset of the kept state or a new allocation), execute (launch to the
 * circuit's completion on the device), download (all 2^n amplitudes into
 * the host complex128 buffer), of which copy wait (waiting on device-to-host
 * copies) and widen (the calling thread's own share of the complex64 ->
 * complex128 conversion)}.  Zeros before the first call.  No counterpart in
 * ket (its run, simulator.cpp:554-558, has no phases to report). */
int ketgpu_run_last_profile(double* out6);
/* Free the device state that ketgpu_run keeps between calls (no-op when
 * there is none).  No counterpart in ket, whose run holds no device memory. */
int ketgpu_release_cache(void);

/* ---- reductions (FP64 accumulation) --------------------------------- */
/* *out = sum over x of |amplitude x|^2 (the squared norm). */
int ketgpu_norm(const ketgpu_state* s, double* out);
/* <a|b> (complex) -- fidelity checks. */
int ketgpu_inner(const ketgpu_state* a, const ketgpu_state* b, double* re, double* im);
/* Compare two states of any precisions: out5 = {max |a_i - b_i| over re and
 * im parts, Re <a|b>, Im <a|b>, <a|a>, <b|b>} (FP64 sums). */
int ketgpu_compare(const ketgpu_state* a, const ketgpu_state* b, double* out5);
/* Replaces ket::expval(State, string) (include/ket/observable.hpp:24,
 * src/observable.cpp:18-83): same masks, same right-to-left order, same
 * errors (length / character -> KETGPU_ERR_INVALID). */
int ketgpu_expval(const ketgpu_state* s, const char* pauli, double* out);
/* Replaces ket::expval(State, PauliSum) (include/ket/observable.hpp:32,
 * src/observable.cpp:85-91); every term in one batched reduction. */
int ketgpu_expval_sum(const ketgpu_state* s, const double* coeffs,
                      const char* const* paulis, uint64_t n_terms, double* out);
/* The value of ketgpu_expval_sum for callers that cannot allocate device
 * memory during the call -- a service that keeps nearly all of HBM reserved
 * for resident states, or code that must not have device memory allocated
 * and freed underneath it.  No counterpart in ket (a variant of this
 * backend's own ketgpu_expval_sum).  It uses a fixed scratch array of
 * 608,256 bytes that every GPU loading the library holds until exit, shared
 * by all calls on that GPU: calls that overlap on one GPU (other streams or
 * threads at the same time) race on it.  The array and this call's kernels
 * are looked up, and so loaded onto the device, when the first state is
 * created there (ketgpu_state_create), which allocates anyway; the call
 * itself allocates nothing.  It synchronises the state's stream and copies
 * the per-term results to the host before returning, so it blocks the host
 * and cannot be used inside stream capture.  At most
 * KETGPU_NOALLOC_MAX_TERMS terms; more returns KETGPU_ERR_INVALID. */
#define KETGPU_NOALLOC_MAX_TERMS 256
int ketgpu_expval_sum_noalloc(const ketgpu_state* s, const double* coeffs,
                              const char* const* paulis, uint64_t n_terms, double* out);
/* Per-term expectations (out has n_terms entries). */
int ketgpu_expval_terms(const ketgpu_state* s, const char* const* paulis,
                        uint64_t n_terms, double* out);

/* ---- sampling: replaces ket::measure (include/ket/measurement.hpp:16-17,
 *      src/measurement.cpp:12-21) ------------------------------------- */
/* The draws ket::measure consumes: uniform_real_distribution<double>(0,1)
 * on std::mt19937{seed}, `count` of them in order. */
int ketgpu_uniforms_mt19937(uint32_t seed, uint64_t count, double* out);
/* Born-rule draws for the given uniforms (host arrays) from one FP64 CDF
 * over a fixed summation tree (segments of 32, carries folded top-down),
 * each draw the first index whose running sum exceeds u.  The tree is kept
 * with the state and rebuilt only after the amplitudes changed (any
 * execute, apply, reset, upload, copy into the state, or
 * ketgpu_state_device_ptr), so repeated draws from one state -- ket's
 * StateVectorSimulation::sample, statevector.cpp:33-42, called once per
 * shot -- cost one descent each. */
int ketgpu_sample(const ketgpu_state* s, const double* uniforms, uint64_t count,
                  uint64_t* out_indices);
/* `count` draws with the uniforms of std::mt19937{seed} +
 * uniform_real_distribution<double>(0,1), in order: the many-shot form of
 * ket::sample (measurement.hpp:26-28 evolves per shot; this draws every shot
 * from one evolution, as the CLI's shot loop would, cli/commands.cpp:159-166). */
int ketgpu_sample_seeded(const ketgpu_state* s, uint32_t seed, uint64_t count,
                         uint64_t* out_indices);
/* Sampling-tree builds since load (all states): a tree is built once per
 * state version.  No counterpart in ket. */
uint64_t ketgpu_sample_tree_builds(void);
/* One draw from std::mt19937{seed} (measurement.cpp:12-21 with a seeded rng). */
int ketgpu_measure(const ketgpu_state* s, uint32_t seed, uint64_t* out_index);

/* ---- adjoint differentiation (no ket counterpart; gradients of
 *      ket::expval(run(circuit(theta)), PauliSum)) ----------------------
 * param_index[i] >= 0 marks op i's first angle as parameter param_index[i]
 * (Rx, Ry, Rz, CRx, CRy, CRz, CP).  params: batch x n_params (row-major);
 * values: batch; grads: batch x n_params.  checkpoint_every > 0 stores the
 * forward state every that many parameterised layers and restarts the
 * reverse sweep's state from the checkpoints. */
int ketgpu_adjoint(int32_t n_qubits, const ketgpu_op* ops, uint64_t n_ops,
                   const int32_t* param_index, const double* params,
                   uint64_t n_params, uint64_t batch, const double* coeffs,
                   const char* const* paulis, uint64_t n_terms,
                   int32_t precision, int32_t checkpoint_every, double* values,
                   double* grads);
/* Sweep methods: AUTO = TILED when n_qubits >= the tile size (12 qubits
 * for KETGPU_C64, 11 for KETGPU_C128), else PER_GATE.  PER_GATE streams the
 * states through HBM once per gate; TILED runs each block of consecutive
 * gates that fits one tile in shared memory and registers, one HBM pass per
 * block.  Both give the same values and gradients up to rounding. */
#define KETGPU_ADJOINT_AUTO 0
#define KETGPU_ADJOINT_PER_GATE 1
#define KETGPU_ADJOINT_TILED 2
/* TILED with each complex64 block's kernel generated with its gates as
 * compile-time constants and compiled at run time (NVRTC, cached per process
 * by block structure; AUTO chooses it for complex64 from 16 qubits).  Falls
 * back to TILED when NVRTC is unavailable. */
#define KETGPU_ADJOINT_TILED_JIT 3
int ketgpu_adjoint_ex(int32_t n_qubits, const ketgpu_op* ops, uint64_t n_ops,
                      const int32_t* param_index, const double* params,
                      uint64_t n_params, uint64_t batch, const double* coeffs,
                      const char* const* paulis, uint64_t n_terms,
                      int32_t precision, int32_t checkpoint_every,
                      int32_t method, double* values, double* grads);
/* NVRTC availability, distinct per-block kernels compiled so far, and
 * launches that used one. */
int ketgpu_adjoint_jit_info(int32_t* available, uint64_t* kernels, uint64_t* launches);
/* The tiled sweeps' plan as flat int32 records (layout documented in
 * ket_b200/csrc/adjoint.cu) for the given checkpoint interval (blocks may
 * run across the barrier-delimited layers of one checkpoint segment, never
 * across its ends); *length receives the record count, out may be NULL to
 * query it. */
int ketgpu_adjoint_plan_describe(int32_t n_qubits, const ketgpu_op* ops,
                                 uint64_t n_ops, const int32_t* param_index,
                                 int32_t precision, int32_t checkpoint_every,
                                 int32_t* out, uint64_t capacity, uint64_t* length);

/* ---- learned fusion cost model (48 -> 128 -> 128 -> 1 MLP, BF16 weights,
 *      FP32 accumulation; no ket counterpart) ------------------------- */
#define KETGPU_MLP_IN 48
#define KETGPU_MLP_HIDDEN 128
int ketgpu_mlp_create(uint64_t seed, ketgpu_mlp** out);
int ketgpu_mlp_destroy(ketgpu_mlp* m);
/* Weights as float (W1 128x48, b1 128, W2 128x128, b2 128, w3 128, b3 1). */
int ketgpu_mlp_get_weights(const ketgpu_mlp* m, float* w1, float* b1, float* w2,
                           float* b2, float* w3, float* b3);
int ketgpu_mlp_set_weights(ketgpu_mlp* m, const float* w1, const float* b1,
                           const float* w2, const float* b2, const float* w3,
                           const float* b3);
/* x: batch x 48 host floats -> out: batch predictions. */
int ketgpu_mlp_forward(ketgpu_mlp* m, const float* x, uint64_t batch, float* out);
/* Gradients of the mean squared error (host outputs, FP32). */
int ketgpu_mlp_gradients(ketgpu_mlp* m, const float* x, const float* y,
                         uint64_t batch, float* loss, float* gw1, float* gb1,
                         float* gw2, float* gb2, float* gw3, float* gb3);
/* `steps` Adam steps over (x, y) minibatches drawn by the library. */
int ketgpu_mlp_train(ketgpu_mlp* m, const float* x, const float* y,
                     uint64_t n_samples, uint64_t steps, uint64_t minibatch,
                     float lr, float* final_loss);
/* Attach a model to the learned planner (NULL detaches).  The model's
 * output is log(pass time in microseconds). */
int ketgpu_planner_set_model(ketgpu_mlp* m);
/* The 48 cost-model features of one pass applying `gates` on an
 * n_qubits state: a dense block over the union of their qubits (fused = 1,
 * tensor = 1 for the tcgen05 path) or one gate through its specialised
 * kernel (fused = 0, exactly one gate). */
int ketgpu_block_features(int32_t n_qubits, int32_t precision, const ketgpu_op* gates,
                          uint64_t n_gates, int32_t fused, int32_t tensor, float* out48);
/* The features of pass `index` of a plan (training rows for the model). */
int ketgpu_plan_pass_features(const ketgpu_plan* p, uint64_t index, float* out48);

#ifdef __cplusplus
}
#endif

#endif
