// ref_shim.cpp -- C entry points over ket's public C++ API.
//
// TEST INFRASTRUCTURE ONLY.  Compiled twice by oracle/Makefile:
//   * with the reference's own state-vector translation units
//     (src/simulator.cpp, src/measurement.cpp, src/observable.cpp,
//     src/backends/statevector.cpp) -> oracle/_ref/libket_ref.so, the
//     reference itself, used to pin the C oracle and as the CPU baseline;
//   * with the B200 drop-in translation unit in their place
//     (ket_b200/host/ket_statevector_gpu.cpp) -> oracle/_ref/libket_dropin.so,
//     which shows ket's unchanged API running on the GPU backend.
// Either way the code below only calls ket's public API
// (include/ket/circuit.hpp, simulator.hpp, measurement.hpp, observable.hpp,
// backends/backend.hpp, parallelism.hpp, qasm.hpp, stepper.hpp).
#include <chrono>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <exception>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include <ket/backends/backend.hpp>
#include <ket/circuit.hpp>
#include <ket/measurement.hpp>
#include <ket/observable.hpp>
#include <ket/parallelism.hpp>
#include <ket/qasm.hpp>
#include <ket/simulator.hpp>
#include <ket/state.hpp>
#include <ket/stepper.hpp>

#include "ketsv_oracle.h"

#define SHIM_API extern "C" __attribute__((visibility("default")))

namespace {

thread_local std::string g_err;

// Error codes mirror the exception the reference threw.
int fail(const std::exception& e, int code) {
  g_err = e.what();
  return code;
}

template <class F>
int guard(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::out_of_range& e) {
    return fail(e, -1);
  } catch (const std::invalid_argument& e) {
    return fail(e, -2);
  } catch (const std::logic_error& e) {
    return fail(e, -3);
  } catch (const std::exception& e) {
    return fail(e, -4);
  }
}

ket::Circuit build(int n, const ko_op* ops, std::size_t nops) {
  ket::Circuit c{static_cast<std::size_t>(n)};
  for (std::size_t i = 0; i < nops; ++i) {
    const ko_op& o = ops[i];
    const auto q0 = static_cast<std::size_t>(o.q[0]);
    const auto q1 = static_cast<std::size_t>(o.q[1]);
    const auto q2 = static_cast<std::size_t>(o.q[2]);
    switch (o.type) {
      case KO_H: c.h(q0); break;
      case KO_X: c.x(q0); break;
      case KO_Y: c.y(q0); break;
      case KO_Z: c.z(q0); break;
      case KO_S: c.s(q0); break;
      case KO_SDG: c.sdg(q0); break;
      case KO_T: c.t(q0); break;
      case KO_TDG: c.tdg(q0); break;
      case KO_RX: c.rx(q0, o.p[0]); break;
      case KO_RY: c.ry(q0, o.p[0]); break;
      case KO_RZ: c.rz(q0, o.p[0]); break;
      case KO_U: c.u(q0, o.p[0], o.p[1], o.p[2]); break;
      case KO_CH: c.ch(q0, q1); break;
      case KO_CX: c.cx(q0, q1); break;
      case KO_CY: c.cy(q0, q1); break;
      case KO_CZ: c.cz(q0, q1); break;
      case KO_CRX: c.crx(q0, q1, o.p[0]); break;
      case KO_CRY: c.cry(q0, q1, o.p[0]); break;
      case KO_CRZ: c.crz(q0, q1, o.p[0]); break;
      case KO_CU: c.cu(q0, q1, o.p[0], o.p[1], o.p[2]); break;
      case KO_CP: c.cp(q0, q1, o.p[0]); break;
      case KO_SWAP: c.swap(q0, q1); break;
      case KO_CCX: c.ccx(q0, q1, q2); break;
      case KO_CSWAP: c.cswap(q0, q1, q2); break;
      case KO_MEASURE: c.measure(q0, q1); break;
      case KO_BARRIER: c.barrier(); break;
      case KO_PROBE: c.probe(); break;
      default: throw std::invalid_argument("shim: unsupported op");
    }
  }
  return c;
}

ket::State to_state(int n, const double* amps) {
  const std::size_t dim = std::size_t{1} << n;
  ket::State s(dim, ket::Complex{0.0, 0.0});
  for (std::size_t i = 0; i < dim; ++i) s[i] = {amps[2 * i], amps[2 * i + 1]};
  return s;
}

void from_state(const ket::State& s, double* out) {
  for (std::size_t i = 0; i < s.size(); ++i) {
    out[2 * i] = s[i].real();
    out[2 * i + 1] = s[i].imag();
  }
}

ket::Method method_of(int m) {
  switch (m) {
    case 1: return ket::Method::StateVector;
    case 2: return ket::Method::Stabilizer;
    default: return ket::Method::Auto;
  }
}

}  // namespace

SHIM_API const char* ref_last_error() { return g_err.c_str(); }

SHIM_API void ref_set_num_threads(unsigned t) { ket::set_num_threads(t); }
SHIM_API unsigned ref_num_threads() { return ket::num_threads(); }

// ket::run (simulator.hpp:15); out holds 2 * 2^n doubles.
SHIM_API int ref_run(int n, const ko_op* ops, std::size_t nops, double* out) {
  return guard([&] { from_state(ket::run(build(n, ops, nops)), out); });
}

// ket::run, timed around the call only (seconds through *secs).
SHIM_API int ref_run_timed(int n, const ko_op* ops, std::size_t nops,
                           double* secs, double* amp0) {
  return guard([&] {
    const ket::Circuit c = build(n, ops, nops);
    const auto t0 = std::chrono::steady_clock::now();
    const ket::State s = ket::run(c);
    const auto t1 = std::chrono::steady_clock::now();
    *secs = std::chrono::duration<double>(t1 - t0).count();
    if (amp0) {
      amp0[0] = s[0].real();
      amp0[1] = s[0].imag();
    }
  });
}

// ket::run, timed around the call only, with the returned state copied to
// out (2 * 2^n doubles) after the clock stops.
SHIM_API int ref_run_timed_state(int n, const ko_op* ops, std::size_t nops,
                                 double* secs, double* out) {
  return guard([&] {
    const ket::Circuit c = build(n, ops, nops);
    const auto t0 = std::chrono::steady_clock::now();
    const ket::State s = ket::run(c);
    const auto t1 = std::chrono::steady_clock::now();
    *secs = std::chrono::duration<double>(t1 - t0).count();
    from_state(s, out);
  });
}

// ket::run_with_probes (simulator.hpp:24): final state plus each probe's state
// (probes_out holds n_probes * 2 * 2^n doubles).
SHIM_API int ref_run_with_probes(int n, const ko_op* ops, std::size_t nops,
                                 double* final_out, double* probes_out,
                                 std::size_t max_probes,
                                 std::size_t* n_probes) {
  return guard([&] {
    const ket::ProbeRun r = ket::run_with_probes(build(n, ops, nops));
    from_state(r.final, final_out);
    const std::size_t dim = std::size_t{1} << n;
    *n_probes = r.probes.size();
    for (std::size_t p = 0; p < r.probes.size() && p < max_probes; ++p)
      from_state(r.probes[p].second, probes_out + 2 * dim * p);
  });
}

// ket::expval(State, pauli) (observable.hpp:24).
SHIM_API int ref_expval(int n, const double* amps, const char* pauli,
                        double* out) {
  return guard([&] { *out = ket::expval(to_state(n, amps), std::string(pauli)); });
}

// ket::expval(State, PauliSum) (observable.hpp:32).
SHIM_API int ref_expval_sum(int n, const double* amps, const double* coeffs,
                            const char* const* paulis, std::size_t nterms,
                            double* out) {
  return guard([&] {
    ket::PauliSum h;
    for (std::size_t t = 0; t < nterms; ++t) h.emplace_back(coeffs[t], paulis[t]);
    *out = ket::expval(to_state(n, amps), h);
  });
}

// ket::expval(Circuit, PauliSum, Method) (observable.hpp:40-41).
SHIM_API int ref_expval_circuit(int n, const ko_op* ops, std::size_t nops,
                                const double* coeffs, const char* const* paulis,
                                std::size_t nterms, int method, double* out) {
  return guard([&] {
    ket::PauliSum h;
    for (std::size_t t = 0; t < nterms; ++t) h.emplace_back(coeffs[t], paulis[t]);
    *out = ket::expval(build(n, ops, nops), h, method_of(method));
  });
}

// `shots` calls of ket::measure(State, rng) on one std::mt19937{seed}
// (measurement.hpp:16).
SHIM_API int ref_measure(int n, const double* amps, std::uint32_t seed,
                         std::size_t shots, std::uint64_t* out) {
  return guard([&] {
    const ket::State s = to_state(n, amps);
    std::mt19937 rng{seed};
    for (std::size_t i = 0; i < shots; ++i) out[i] = ket::measure(s, rng);
  });
}

// The uniform stream ket::measure consumes: uniform_real_distribution<double>
// on std::mt19937{seed} (measurement.cpp:13-14).
SHIM_API void ref_uniforms(std::uint32_t seed, std::size_t count, double* out) {
  std::mt19937 rng{seed};
  std::uniform_real_distribution<double> dist(0.0, 1.0);
  for (std::size_t i = 0; i < count; ++i) out[i] = dist(rng);
}

// `shots` calls of ket::sample(Circuit, rng, method) (measurement.hpp:26-28);
// creg_out holds shots * n_clbits ints.
SHIM_API int ref_sample(int n, const ko_op* ops, std::size_t nops,
                        std::uint32_t seed, int method, std::size_t shots,
                        int* creg_out, std::size_t* n_clbits) {
  return guard([&] {
    const ket::Circuit c = build(n, ops, nops);
    std::mt19937 rng{seed};
    *n_clbits = c.n_clbits();
    for (std::size_t s = 0; s < shots; ++s) {
      const std::vector<int> r = ket::sample(c, rng, method_of(method));
      for (std::size_t b = 0; b < r.size(); ++b) creg_out[s * r.size() + b] = r[b];
    }
  });
}

// The same shots through one Simulation (backend.hpp:57): evolve once.
SHIM_API int ref_simulate_sample(int n, const ko_op* ops, std::size_t nops,
                                 std::uint32_t seed, int method,
                                 std::size_t shots, int* creg_out,
                                 std::size_t* n_clbits, char* backend_name,
                                 std::size_t name_len) {
  return guard([&] {
    const ket::Circuit c = build(n, ops, nops);
    const auto sim = ket::simulate(c, method_of(method));
    std::mt19937 rng{seed};
    *n_clbits = c.n_clbits();
    for (std::size_t s = 0; s < shots; ++s) {
      const std::vector<int> r = sim->sample(rng);
      for (std::size_t b = 0; b < r.size(); ++b) creg_out[s * r.size() + b] = r[b];
    }
    if (backend_name && name_len) {
      const std::string_view nm = sim->backend();
      const std::size_t k = nm.size() < name_len - 1 ? nm.size() : name_len - 1;
      std::memcpy(backend_name, nm.data(), k);
      backend_name[k] = '\0';
    }
  });
}

// ket::is_clifford / ket::chosen_method (backend.hpp:48-52).
SHIM_API int ref_is_clifford(int n, const ko_op* ops, std::size_t nops,
                             int* out) {
  return guard([&] { *out = ket::is_clifford(build(n, ops, nops)) ? 1 : 0; });
}

SHIM_API int ref_chosen_method(int n, const ko_op* ops, std::size_t nops,
                               int* out) {
  return guard([&] {
    *out = ket::chosen_method(build(n, ops, nops)) == ket::Method::Stabilizer ? 2 : 1;
  });
}

namespace {

// A parsed circuit's gates with composites expanded through their wire map
// (as simulator.cpp:504-511 expands them), one ko_op each.  A barrier keeps
// its qubit count in nq and its first three qubits in q; a measure keeps its
// classical bit in q[1].
void flatten(const ket::Circuit& c, const std::vector<std::size_t>& wire, std::vector<ko_op>& out) {
  for (const ket::DagNode& node : c.dag().nodes()) {
    const ket::Gate& g = node.gate;
    if (g.type == ket::GateType::Composite) {
      if (!g.definition) continue;
      std::vector<std::size_t> sub;
      for (const auto& q : g.qubits) sub.push_back(wire[q.index]);
      flatten(*g.definition, sub, out);
      continue;
    }
    ko_op o{};
    o.type = static_cast<int32_t>(g.type);
    o.nq = static_cast<int32_t>(g.qubits.size());
    for (std::size_t k = 0; k < g.qubits.size() && k < 3; ++k)
      o.q[k] = static_cast<int32_t>(wire[g.qubits[k].index]);
    if (g.type == ket::GateType::Measure) o.q[1] = static_cast<int32_t>(g.clbit);
    for (std::size_t k = 0; k < g.params.size() && k < 3; ++k) o.p[k] = g.params[k];
    out.push_back(o);
  }
}

}  // namespace

// ket::from_qasm (bindings/qasm/qasm.cpp:479-544), flattened: the register
// sizes, the number of top-level nodes and up to cap ops (n_out = all).
SHIM_API int ref_qasm_parse(const char* src, int* n_qubits, int* n_clbits, int* n_top, ko_op* out,
                            std::size_t cap, std::size_t* n_out) {
  return guard([&] {
    const ket::Circuit c = ket::from_qasm(src);
    std::vector<std::size_t> wire(c.n_qubits());
    for (std::size_t i = 0; i < wire.size(); ++i) wire[i] = i;
    std::vector<ko_op> ops;
    flatten(c, wire, ops);
    *n_qubits = static_cast<int>(c.n_qubits());
    *n_clbits = static_cast<int>(c.n_clbits());
    *n_top = static_cast<int>(c.dag().nodes().size());
    for (std::size_t i = 0; i < ops.size() && i < cap; ++i) out[i] = ops[i];
    *n_out = ops.size();
  });
}

// ket::to_qasm(ket::from_qasm(src)) (qasm.cpp:764-780) into buf; len = the
// full length, of which min(len, cap - 1) bytes and a terminator are written.
SHIM_API int ref_qasm_roundtrip(const char* src, char* buf, std::size_t cap, std::size_t* len) {
  return guard([&] {
    const std::string text = ket::to_qasm(ket::from_qasm(src));
    *len = text.size();
    if (cap > 0) {
      const std::size_t n = text.size() < cap - 1 ? text.size() : cap - 1;
      std::memcpy(buf, text.data(), n);
      buf[n] = '\0';
    }
  });
}

// ket::to_qasm of a circuit built from flat ops (no composites).
SHIM_API int ref_to_qasm(int n, const ko_op* ops, std::size_t nops, char* buf, std::size_t cap,
                         std::size_t* len) {
  return guard([&] {
    const std::string text = ket::to_qasm(build(n, ops, nops));
    *len = text.size();
    if (cap > 0) {
      const std::size_t k = text.size() < cap - 1 ? text.size() : cap - 1;
      std::memcpy(buf, text.data(), k);
      buf[k] = '\0';
    }
  });
}

// ket::State::print (src/state.cpp:42-52) of 2^n amplitudes.
SHIM_API int ref_state_print(int n, const double* amps, char* buf, std::size_t cap, std::size_t* len) {
  return guard([&] {
    const std::string text = to_state(n, amps).print();
    *len = text.size();
    if (cap > 0) {
      const std::size_t k = text.size() < cap - 1 ? text.size() : cap - 1;
      std::memcpy(buf, text.data(), k);
      buf[k] = '\0';
    }
  });
}

// ket::Stepper (include/ket/stepper.hpp:18-41) stepped to the end: the state
// at every position 0..size() into out (up to cap states of 2^n amplitudes),
// n_steps = size().  A step() past the end must return false.
SHIM_API int ref_stepper_walk(int n, const ko_op* ops, std::size_t nops, double* out, std::size_t cap,
                              std::size_t* n_steps) {
  return guard([&] {
    ket::Stepper s{build(n, ops, nops)};
    *n_steps = s.size();
    const std::size_t dim = std::size_t{1} << n;
    std::size_t k = 0;
    const auto record = [&] {
      if (k < cap) from_state(s.state(), out + 2 * dim * k);
      ++k;
    };
    record();
    while (s.step()) record();
    if (!s.at_end() || s.step()) throw std::logic_error("stepper: stepped past the end");
  });
}

// ket::Stepper::seek(k) for each k of seq in turn: the state after each
// (n_seq states of 2^n amplitudes) and pos() after each.
SHIM_API int ref_stepper_seek(int n, const ko_op* ops, std::size_t nops, const std::size_t* seq,
                              std::size_t n_seq, double* out, std::size_t* pos) {
  return guard([&] {
    ket::Stepper s{build(n, ops, nops)};
    const std::size_t dim = std::size_t{1} << n;
    for (std::size_t i = 0; i < n_seq; ++i) {
      s.seek(seq[i]);
      pos[i] = s.pos();
      from_state(s.state(), out + 2 * dim * i);
    }
  });
}
