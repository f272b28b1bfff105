// ket_statevector_gpu.cpp -- ket's state-vector translation units, re-done on
// the B200 backend.
//
// A ket build that links this file instead of src/simulator.cpp,
// src/measurement.cpp, src/observable.cpp and src/backends/statevector.cpp
// keeps ket's public API unchanged (include/ket/simulator.hpp,
// measurement.hpp, observable.hpp, stepper.hpp) while every state-vector
// computation runs in libket_b200.so.  Auto routing is untouched: ket's own
// simulate() (src/backends/backend.cpp:54-70) still sends Clifford circuits
// to its CPU stabilizer tableau and reaches the GPU only through
// make_statevector_simulation (src/backends/internal.hpp:33).
//
// Options come from the environment: KET_B200_PRECISION = c128 (default) |
// c64, KET_B200_FUSION = greedy (default) | none | reference | learned,
// KET_B200_MAX_K = 1..6 (default 5), KET_B200_TENSOR = 1 (default) | 0.
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <string_view>
#include <utility>
#include <vector>

#include <ket/backends/backend.hpp>
#include <ket/circuit.hpp>
#include <ket/dag.hpp>
#include <ket/gate.hpp>
#include <ket/measurement.hpp>
#include <ket/observable.hpp>
#include <ket/simulator.hpp>
#include <ket/state.hpp>
#include <ket/stepper.hpp>

#include "internal.hpp"  // ket's src/backends/internal.hpp (the backend seam)
#include "ket_b200.h"

namespace ket {
namespace {

// KETGPU_ERR_* -> the exception ket throws for the same condition.
void check(int rc) {
  if (rc == KETGPU_OK) return;
  const std::string msg = ketgpu_last_error();
  if (rc == KETGPU_ERR_OUT_OF_RANGE) throw std::out_of_range(msg);
  if (rc == KETGPU_ERR_INVALID) throw std::invalid_argument(msg);
  if (rc == KETGPU_ERR_LOGIC) throw std::logic_error(msg);
  throw std::runtime_error(msg);
}

ketgpu_options options() {
  ketgpu_options o{KETGPU_C128, KETGPU_FUSE_GREEDY, 0, 1, 0};  // k: the library default
  if (const char* p = std::getenv("KET_B200_PRECISION"))
    o.precision = std::string(p) == "c64" ? KETGPU_C64 : KETGPU_C128;
  if (const char* f = std::getenv("KET_B200_FUSION")) {
    const std::string s(f);
    o.fusion = s == "none" ? KETGPU_FUSE_NONE
               : s == "reference" ? KETGPU_FUSE_REFERENCE
               : s == "learned" ? KETGPU_FUSE_LEARNED
                                : KETGPU_FUSE_GREEDY;
  }
  if (const char* k = std::getenv("KET_B200_MAX_K")) o.max_block_qubits = std::atoi(k);
  if (const char* t = std::getenv("KET_B200_TENSOR")) o.tensor_cores = std::atoi(t) != 0;
  return o;
}

// Flatten the DAG in insertion order, remapping composite blocks' wires as
// ket's apply_circuit does (src/simulator.cpp:482-517).  Probes are kept so
// run_with_probes can split at them.
void flatten(const Circuit& c, const std::vector<std::size_t>& wire, std::vector<ketgpu_op>& out,
             std::vector<std::string>* probe_labels) {
  for (const DagNode& node : c.dag().nodes()) {
    const Gate& g = node.gate;
    if (g.type == GateType::Composite) {
      std::vector<std::size_t> sub(g.definition->n_qubits());
      for (std::size_t j = 0; j < g.qubits.size(); ++j) sub[j] = wire[g.qubits[j].index];
      flatten(*g.definition, sub, out, probe_labels);
      continue;
    }
    ketgpu_op op{};
    op.type = static_cast<int32_t>(g.type);
    if (g.type == GateType::Barrier || g.type == GateType::Probe) {
      if (g.type == GateType::Probe && probe_labels) probe_labels->push_back(g.label);
      out.push_back(op);
      continue;
    }
    op.nq = static_cast<int32_t>(g.qubits.size());
    for (std::size_t j = 0; j < g.qubits.size() && j < 3; ++j)
      op.q[j] = static_cast<int32_t>(wire[g.qubits[j].index]);
    if (g.type == GateType::Measure) op.q[1] = static_cast<int32_t>(g.clbit);
    for (std::size_t j = 0; j < g.params.size() && j < 3; ++j) op.p[j] = g.params[j];
    out.push_back(op);
  }
}

std::vector<ketgpu_op> ops_of(const Circuit& c, std::vector<std::string>* probes = nullptr) {
  std::vector<std::size_t> wire(c.n_qubits());
  for (std::size_t i = 0; i < wire.size(); ++i) wire[i] = i;
  std::vector<ketgpu_op> ops;
  flatten(c, wire, ops, probes);
  return ops;
}

// An owned device state.
struct DeviceState {
  ketgpu_state* h = nullptr;
  DeviceState(std::size_t n, int precision) {
    check(ketgpu_state_create(static_cast<int32_t>(n), precision, &h));
  }
  ~DeviceState() {
    if (h) ketgpu_state_destroy(h);
  }
  DeviceState(const DeviceState&) = delete;
  DeviceState& operator=(const DeviceState&) = delete;
  void apply(const std::vector<ketgpu_op>& ops, const ketgpu_options& o) {
    check(ketgpu_apply(h, ops.data(), ops.size(), &o));
  }
  State to_host(std::size_t n) const {
    State s(std::size_t{1} << n, Complex{0.0, 0.0});
    check(ketgpu_state_download(h, 0, s.size(), reinterpret_cast<double*>(&s[0])));
    return s;
  }
  static std::unique_ptr<DeviceState> from_host(const State& s) {
    std::size_t n = 0;
    while ((std::size_t{1} << n) < s.size()) ++n;
    if ((std::size_t{1} << n) != s.size()) throw std::invalid_argument("state size is not a power of two");
    auto d = std::make_unique<DeviceState>(n, KETGPU_C128);
    check(ketgpu_state_upload(d->h, 0, s.size(), reinterpret_cast<const double*>(&s[0])));
    return d;
  }
};

std::size_t draw(const DeviceState& d, std::mt19937& rng) {
  std::uniform_real_distribution<double> dist(0.0, 1.0);  // measurement.cpp:13-14
  const double u = dist(rng);
  uint64_t out = 0;
  check(ketgpu_sample(d.h, &u, 1, &out));
  return static_cast<std::size_t>(out);
}

double pauli_sum_on(const DeviceState& d, const PauliSum& h) {
  std::vector<double> coeffs;
  std::vector<const char*> paulis;
  for (const auto& [c, p] : h) {
    coeffs.push_back(c);
    paulis.push_back(p.c_str());
  }
  double out = 0.0;
  check(ketgpu_expval_sum(d.h, coeffs.data(), paulis.data(), paulis.size(), &out));
  return out;
}

// The GPU-resident StateVector backend (replaces statevector.cpp:26-51): the
// circuit is evolved once into HBM; samples and expectations are answered
// there, and the 2^n vector never crosses to the host.
class GpuStateVectorSimulation final : public Simulation {
 public:
  explicit GpuStateVectorSimulation(const Circuit& circuit)
      : opt_(options()),
        state_(circuit.n_qubits(), opt_.precision),
        measurements_(collect_measurements(circuit)) {
    state_.apply(ops_of(circuit), opt_);
  }
  std::string_view backend() const override { return "state vector"; }
  std::vector<int> sample(std::mt19937& rng) const override {
    const std::size_t outcome = draw(state_, rng);
    std::vector<int> creg(measurements_.n_clbits, 0);
    for (const MeasuredBit& m : measurements_.bits)
      creg[m.clbit] = static_cast<int>((outcome >> m.qubit) & 1u);
    return creg;
  }
  double expval(const std::string& pauli) const override {
    double out = 0.0;
    check(ketgpu_expval(state_.h, pauli.c_str(), &out));
    return out;
  }
  // Every term of a Pauli sum in one batched reduction over the kept state.
  double expval_sum(const PauliSum& h) const { return pauli_sum_on(state_, h); }

 private:
  ketgpu_options opt_;
  DeviceState state_;
  Measurements measurements_;
};

State ground(std::size_t n) {
  State s(std::size_t{1} << n, Complex{0.0, 0.0});
  s[0] = Complex{1.0, 0.0};
  return s;
}

}  // namespace

// ---- simulator.hpp ---------------------------------------------------------
State run(const Circuit& circuit) {
  const std::vector<ketgpu_op> ops = ops_of(circuit);
  const ketgpu_options o = options();
  State s(std::size_t{1} << circuit.n_qubits(), Complex{0.0, 0.0});
  check(ketgpu_run(static_cast<int32_t>(circuit.n_qubits()), ops.data(), ops.size(), &o,
                   reinterpret_cast<double*>(&s[0])));
  return s;
}

ProbeRun run_with_probes(const Circuit& circuit) {
  std::vector<std::string> labels;
  const std::vector<ketgpu_op> ops = ops_of(circuit, &labels);
  const ketgpu_options o = options();
  DeviceState d(circuit.n_qubits(), o.precision);
  std::vector<std::pair<std::string, State>> probes;
  std::vector<ketgpu_op> seg;
  std::size_t pi = 0;
  for (const ketgpu_op& op : ops) {
    if (op.type == static_cast<int32_t>(GateType::Probe)) {
      d.apply(seg, o);
      seg.clear();
      probes.emplace_back(labels[pi++], d.to_host(circuit.n_qubits()));
    } else {
      seg.push_back(op);
    }
  }
  d.apply(seg, o);
  return ProbeRun{d.to_host(circuit.n_qubits()), std::move(probes)};
}

// ---- measurement.hpp -------------------------------------------------------
std::size_t measure(const State& state, std::mt19937& rng) {
  return draw(*DeviceState::from_host(state), rng);
}

std::size_t measure(const State& state) {
  thread_local std::mt19937 rng{std::random_device{}()};
  return measure(state, rng);
}

std::vector<int> sample(const Circuit& circuit, std::mt19937& rng, Method method) {
  return simulate(circuit, method)->sample(rng);
}

std::vector<int> sample(const Circuit& circuit, Method method) {
  thread_local std::mt19937 rng{std::random_device{}()};
  return sample(circuit, rng, method);
}

// ---- observable.hpp --------------------------------------------------------
double expval(const State& state, const std::string& pauli) {
  const auto d = DeviceState::from_host(state);
  double out = 0.0;
  check(ketgpu_expval(d->h, pauli.c_str(), &out));
  return out;
}

double expval(const State& state, const PauliSum& hamiltonian) {
  return pauli_sum_on(*DeviceState::from_host(state), hamiltonian);
}

double expval(const Circuit& circuit, const std::string& pauli, Method method) {
  return simulate(circuit, method)->expval(pauli);
}

double expval(const Circuit& circuit, const PauliSum& hamiltonian, Method method) {
  const std::unique_ptr<Simulation> sim = simulate(circuit, method);
  // On the GPU every term is reduced in one launch; the coefficient-weighted
  // sum is still taken in term order (observable.cpp:97-106 loops the terms).
  if (const auto* gpu = dynamic_cast<const GpuStateVectorSimulation*>(sim.get()))
    return gpu->expval_sum(hamiltonian);
  double total = 0.0;
  for (const auto& [coeff, pauli] : hamiltonian) total += coeff * sim->expval(pauli);
  return total;
}

// ---- backends/internal.hpp seam ------------------------------------------
std::unique_ptr<Simulation> make_statevector_simulation(const Circuit& circuit) {
  return std::make_unique<GpuStateVectorSimulation>(circuit);
}

// ---- stepper.hpp -----------------------------------------------------------
// One DAG node per step, applied on the GPU.  ket's header makes
// Stepper::state() an inline read of the host member state_, so the host
// copy must be current after every step; what stays on the device is the
// state the next step starts from.  The device copy of the Stepper that moved
// last is kept (one at a time: ket's Stepper has no destructor of ours, so
// this bounds what a destroyed Stepper can leave behind), tagged with its
// address, its host buffer and position; a step that finds another tag
// uploads state_ first.  Each step then costs its gates plus one download,
// instead of an upload and a download.
namespace {

struct StepperDevice {
  std::mutex mu;
  const Stepper* owner = nullptr;
  const void* host = nullptr;  // address of the owner's first amplitude when the copy was made
  std::size_t pos = 0, n = 0;
  std::unique_ptr<DeviceState> dev;
};

StepperDevice& stepper_device() {
  static StepperDevice d;
  return d;
}

std::vector<ketgpu_op> node_ops(const Circuit& c, std::size_t from, std::size_t to) {
  std::vector<ketgpu_op> ops;
  for (std::size_t i = from; i < to; ++i) {
    const Gate& g = c.dag().nodes()[i].gate;
    if (g.type == GateType::Measure || g.type == GateType::Barrier || g.type == GateType::Probe) continue;
    if (g.type == GateType::Composite) {
      std::vector<std::size_t> sub(g.definition->n_qubits());
      for (std::size_t j = 0; j < g.qubits.size(); ++j) sub[j] = g.qubits[j].index;
      flatten(*g.definition, sub, ops, nullptr);
    } else {
      ketgpu_op op{};
      op.type = static_cast<int32_t>(g.type);
      op.nq = static_cast<int32_t>(g.qubits.size());
      for (std::size_t j = 0; j < g.qubits.size() && j < 3; ++j) op.q[j] = static_cast<int32_t>(g.qubits[j].index);
      for (std::size_t j = 0; j < g.params.size() && j < 3; ++j) op.p[j] = g.params[j];
      ops.push_back(op);
    }
  }
  return ops;
}

// Apply DAG nodes [from, to) of `c` to `state` (the Stepper `who` at
// position `from`), leaving the result in `state` and on the device.
void advance(const Stepper* who, State& state, const Circuit& c, std::size_t from, std::size_t to) {
  const std::vector<ketgpu_op> ops = node_ops(c, from, to);
  StepperDevice& sd = stepper_device();
  std::lock_guard<std::mutex> lk(sd.mu);
  const bool mine = sd.dev && sd.owner == who && sd.host == static_cast<const void*>(&state[0]) && sd.pos == from &&
                    sd.n == c.n_qubits();
  if (ops.empty()) {  // structural nodes only: the state does not change
    if (mine) sd.pos = to;
    return;
  }
  if (!mine) {
    sd.owner = nullptr;
    sd.dev.reset();
    sd.dev = DeviceState::from_host(state);
  }
  ketgpu_options o = options();
  o.precision = KETGPU_C128;
  o.fusion = KETGPU_FUSE_NONE;  // the stepper's semantics: one node at a time
  sd.dev->apply(ops, o);
  check(ketgpu_state_download(sd.dev->h, 0, state.size(), reinterpret_cast<double*>(&state[0])));
  sd.owner = who;
  sd.host = &state[0];
  sd.pos = to;
  sd.n = c.n_qubits();
}

}  // namespace

Stepper::Stepper(Circuit circuit)
    : circuit_(std::move(circuit)),
      state_(ground(circuit_.n_qubits())),
      n_steps_(circuit_.dag().nodes().size()),
      pos_(0) {}

void Stepper::reset() {
  state_ = ground(circuit_.n_qubits());
  pos_ = 0;
}

bool Stepper::step() {
  if (pos_ >= n_steps_) return false;
  advance(this, state_, circuit_, pos_, pos_ + 1);
  ++pos_;
  return true;
}

void Stepper::seek(std::size_t step) {
  if (step > n_steps_) step = n_steps_;
  if (step < pos_) reset();
  advance(this, state_, circuit_, pos_, step);
  pos_ = step;
}

}  // namespace ket
