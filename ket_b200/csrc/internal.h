// internal.h -- shared host-side declarations of the B200 state-vector
// backend (not installed; the public surface is include/ket_b200.h).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <complex>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ket_b200.h"

namespace kb {

using cplx = std::complex<double>;

// ---- errors ----------------------------------------------------------------
// Thrown inside the library, turned into KETGPU_ERR_* at the ABI boundary.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
[[noreturn]] void fail(int code, const std::string& msg);
void check_cuda(cudaError_t e, const char* what);
void set_last_error(const char* msg);
#define KB_CUDA(x) ::kb::check_cuda((x), #x)

extern std::atomic<uint64_t> g_launches;
inline void count_launch(uint64_t k = 1) { g_launches.fetch_add(k, std::memory_order_relaxed); }

// Switch to a device for the lifetime of the guard.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev);
  ~DeviceGuard();
};

// ---- state -----------------------------------------------------------------
struct State {
  int n = 0;
  int precision = KETGPU_C64;
  int device = 0;
  void* amps = nullptr;  // float2[2^n] or double2[2^n]
  cudaStream_t stream = nullptr;
  // Bumped by every write the library makes to the amplitudes (touch()).
  mutable uint64_t version = 0;
  // The sampling tree (FP64 level sums with folded carries) of the state at
  // tree_version, kept for the next draws; built by sample_tree on demand.
  mutable double* tree = nullptr;
  mutable uint64_t tree_doubles = 0;
  mutable uint64_t tree_version = ~uint64_t{0};
  // version right after set_ground: while version still equals it, the state
  // is |0...0> and its squared norm is exactly 1
  mutable uint64_t ground_version = ~uint64_t{0};
  uint64_t dim() const { return uint64_t{1} << n; }
  size_t amp_bytes() const { return precision == KETGPU_C64 ? 8 : 16; }
  void touch() const { ++version; }
};

// ---- passes ----------------------------------------------------------------
// One kernel launch of a plan.
enum class PassKind : int {
  Pair,      // 2x2 on (k0, k1) = (base|P0, base|P1), base ranges over the
             // indices with zeros at the fixed positions
  Phase,     // multiply the amplitudes with all fixed bits set by a phase
  Fused,     // dense 2^k x 2^k complex matrix on k qubits
  NormCapture,  // record the state's squared norm (FP64) on the device
  NormRestore,  // rescale the state to the recorded squared norm
  Diagonal,     // multiply amplitude x by exp(i phi(x)), phi a quadratic
                // polynomial in the index bits (a run of diagonal gates)
  SharedRun,    // consecutive gates on qubits below kRunBits, applied one
                // after another to chunks of 2^kRunBits amplitudes held in
                // shared memory (one HBM pass for the run)
};
// Chunk bits of a shared-memory run: its gates act on qubits 0..kRunBits-1.
constexpr int kRunBits = 11;
constexpr int kRunMaxGates = 128;
enum PairMode : int { kPairGeneral = 0, kPairSwap = 1, kPairDiag = 2 };

struct Pass {
  PassKind kind = PassKind::Pair;
  int mode = kPairGeneral;
  int nfixed = 0;
  int fixed[3] = {0, 0, 0};  // sorted ascending
  uint64_t p0 = 0, p1 = 0;   // bit patterns of element 0 / element 1
  cplx m[4];                 // 2x2 (Pair) ; m[0] = phase (Phase)
  // Fused
  int k = 0;
  int qubits[6] = {0, 0, 0, 0, 0, 0};  // sorted ascending; matrix bit b <-> qubits[b]
  size_t mat_index = 0;                // into Plan::matrices
  bool tensor = false;                 // tcgen05 path
  // tcgen05 block directly before the plan's NormRestore: it also writes
  // per-CTA FP64 sums of |out|^2 into the plan's norm partials, and the
  // restore (norm_out set there too) takes the norm from them
  bool norm_out = false;
  size_t diag_index = 0;               // Diagonal: into Plan::diags
  size_t run_index = 0;                // SharedRun: into Plan::runs
  int first_op = 0, n_gates = 0;       // provenance
  std::vector<int> gates;              // op indices of the gates this pass applies
  double bytes(int n, size_t amp) const;
};

// Phase polynomial of a run of diagonal gates: the amplitude with index bits
// x_0..x_{n-1} is multiplied by exp(i phi(x)),
//   phi(x) = c0 + sum_i a[i] x_i + sum_{i<j} b[i*n + j] x_i x_j.
struct DiagPoly {
  double c0 = 0.0;
  std::vector<double> a;  // n
  std::vector<double> b;  // n x n, upper triangle used
};
// Low index bits whose pair terms are tabulated by the diagonal kernel.
constexpr int kDiagLowBits = 12;

struct Plan {
  int n = 0;
  int precision = KETGPU_C64;
  std::vector<ketgpu_op> ops;  // the circuit the plan was built from
  std::vector<Pass> passes;
  std::vector<std::vector<cplx>> matrices;  // FP64 block matrices (host)
  // device copies, built lazily per device: FP64 (c128 SIMT), FP32 (c64 SIMT),
  // tcgen05 B operands (hi/lo fp16 images in the shared-memory layout)
  void* d_mat64 = nullptr;
  void* d_mat32 = nullptr;
  void* d_tc = nullptr;
  double* d_norm = nullptr;  // [captured, current, block partials...]
  std::vector<DiagPoly> diags;  // Diagonal passes (host)
  void* d_diag = nullptr;       // per Diagonal pass: low-bit table + coefficients
  std::vector<std::vector<Pass>> runs;  // SharedRun passes: each gate lowered (host)
  void* d_runs = nullptr;               // their device gate records
  std::vector<size_t> off64, off32, offtc, offdiag, offrun;
  int device = -1;
  ketgpu_plan_stats stats{};
  ~Plan();
};

// ---- gate lowering -----------------------------------------------------------
bool is_unitary(int type);
int gate_arity(int type);
void validate_ops(int n, const ketgpu_op* ops, uint64_t nops);
// The 2x2 matrix of a 1-qubit gate (or the target block of a controlled
// rotation), built with ket's formulas (simulator.cpp:38-97, 166-200).
void single_matrix(int type, const double* p, cplx m[4]);
// Lower one gate to its specialised pass.
Pass lower_gate(const ketgpu_op& op);
// Per-gate cost in state passes (fraction of the state each pass moves).
double gate_traffic_fraction(const ketgpu_op& op);
// Dense block matrix of a gate list restricted to `qubits` (bit b <-> qubits[b]).
std::vector<cplx> block_matrix(const std::vector<const ketgpu_op*>& gates,
                               const int* qubits, int k);

// ---- planner ---------------------------------------------------------------
struct PlanOptions {
  int precision = KETGPU_C64;
  int fusion = KETGPU_FUSE_GREEDY;
  int max_k = 5;
  bool tensor = true;
  int renormalize = 0;
};
constexpr int kNormBlocks = 592;  // 4 x 148 SMs
PlanOptions resolve_options(const ketgpu_options* opt);
void build_plan(Plan& plan, int n, const ketgpu_op* ops, uint64_t nops,
                const PlanOptions& o);
// Cost-model features of one pass: a dense block over `qubits` (fused) or
// one gate through its specialised kernel (gates.size() == 1, !fused).
constexpr int kFeatures = 48;
void pass_features(int n, int precision, const std::vector<const ketgpu_op*>& gates,
                   const std::vector<int>& qubits, bool fused, bool tensor, float* out);
// Learned-planner hooks (mlp.cu): the attached model, and batched
// predictions of pass times (microseconds) for feature rows.
bool learned_model_attached();
void learned_predict(const std::vector<float>& rows, std::vector<float>& us);

// ---- kernel launchers (gates.cu / fused_tc.cu / reduce.cu) -----------------
void launch_pass(const State& s, const Plan& plan, const Pass& p);
void upload_plan_matrices(Plan& plan, int device);
// norm_partials: null, or kNormBlocks doubles that receive the per-CTA sums
// of |out|^2 (zero beyond the grid).
void launch_fused_tc(const State& s, const Pass& p, const void* b_image, double* norm_partials = nullptr);
// Host only: the producer and epilogue forms a tensor-core launch of pass p
// on an n-qubit state takes (tma_dims = tensor-map dimensions, 0 for the
// cp.async producers; direct = register-to-HBM stores), given the tensor-map
// encoder of the driver.
void tc_form(int n, const Pass& p, int* tma_dims, int* direct);
// Diagonal pass: device data = table (2^L complex, state precision) then FP64
// coefficients, laid out by diag_device_data (diag.cu).
void launch_diag(const State& s, const Pass& p, const void* data);
// SharedRun pass: device gate records laid out by run_device_data (gates.cu).
void launch_run(const State& s, const Pass& p, const void* data);
void run_device_data(const std::vector<Pass>& gates, int precision, std::vector<unsigned char>& out);
void diag_device_data(const DiagPoly& poly, int n, int precision, std::vector<unsigned char>& out);
bool is_diagonal_gate(int type);
// Add one diagonal gate's phase terms to a polynomial.
void add_diagonal_gate(const ketgpu_op& op, DiagPoly& poly, int n);
// Size in bytes of one tcgen05 B image for a k-qubit block.
size_t tc_image_bytes(int k);
void build_tc_image(const std::vector<cplx>& mat, int k, std::vector<uint32_t>& out);
bool tc_supported(int k);

void set_ground(const State& s);
// Squared norm into a device scalar (partials: kNormBlocks doubles).
void norm_to_device(const State& s, double* partials, double* out);
// The same from partials a tensor-core block already wrote (in index order).
void norm_from_partials(const State& s, const double* partials, double* out);
// Look up (and so load) the no-allocation entry point's scratch array and
// kernels on `device`, which must be current; once per device, at the first
// state created there.
void noalloc_prepare(int device);
// Free the device state that ketgpu_run keeps between calls (if any).
void release_run_state();
// s *= sqrt(target[0] / current[0]), factor read on the device.
void rescale_state(const State& s, const double* target, const double* current);
double reduce_norm(const State& s);
cplx reduce_inner(const State& a, const State& b);
void compare_states(const State& a, const State& b, double out[5]);
void expval_terms(const State& s, const std::vector<uint64_t>& flip,
                  const std::vector<uint64_t>& sign, const std::vector<int>& phase,
                  double* out);
// Born-rule draws for host uniforms; builds the state's sampling tree only
// when the amplitudes changed since the last build (State::version).
void sample_tree(const State& s, const double* u, uint64_t count, uint64_t* out);
// Number of sampling-tree builds since load (all states).
uint64_t sample_tree_builds();

// Pauli-string masks (observable.cpp:68-113); throws Error(INVALID).
void pauli_masks(int n, const char* pauli, uint64_t& flip, uint64_t& sign, int& phase_q);

}  // namespace kb
