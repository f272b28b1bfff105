"""ctypes front-end for the CPU checkers (test infrastructure only).

* ``Oracle`` wraps ``oracle/_build/libketsv_oracle.so``, the plain-C
  restatement of ket's state-vector algorithm (see ketsv_oracle.c for the
  reference file:line of every function).
* ``Reference`` wraps ``oracle/_ref/libket_ref.so``: ket itself, compiled from
  its own sources by ``oracle/Makefile``, called through its public C++ API
  (``ref_shim.cpp``).  ``Reference(dropin=True)`` loads the same shim linked
  against the B200 drop-in unit instead of ket's state-vector units.

Only the tests, the smoke check and the benchmark's CPU-baseline leg import
this module; the product (``ket_b200``) never does.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libketsv_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libket_ref.so")
DROPIN_SO = os.path.join(HERE, "_ref", "libket_dropin.so")

# 48-byte flat op, identical to ko_op / ketgpu_op.
OP_DTYPE = np.dtype([("type", "<i4"), ("nq", "<i4"), ("q", "<i4", (3,)),
                     ("aux", "<i4"), ("p", "<f8", (3,))], align=True)
assert OP_DTYPE.itemsize == 48

GATES = ["H", "X", "Y", "Z", "S", "Sdg", "T", "Tdg", "Rx", "Ry", "Rz", "U",
         "CH", "CX", "CY", "CZ", "CRx", "CRy", "CRz", "CU", "CP", "Swap",
         "CCX", "CSwap", "Measure", "Barrier", "Composite", "Probe"]
CODE = {g: i for i, g in enumerate(GATES)}
ARITY = {g: (1 if i <= 11 else 2 if i <= 21 else 3 if i <= 23 else 0)
         for i, g in enumerate(GATES)}
NPARAMS = {"Rx": 1, "Ry": 1, "Rz": 1, "U": 3, "CRx": 1, "CRy": 1, "CRz": 1,
           "CU": 3, "CP": 1}


def make_ops(gates):
    """[(name, qubits, params)] -> numpy array of OP_DTYPE."""
    ops = np.zeros(len(gates), dtype=OP_DTYPE)
    for i, g in enumerate(gates):
        name, qubits = g[0], g[1]
        params = g[2] if len(g) > 2 else ()
        ops[i]["type"] = CODE[name]
        ops[i]["nq"] = len(qubits)
        for j, q in enumerate(qubits):
            ops[i]["q"][j] = q
        for j, v in enumerate(params):
            ops[i]["p"][j] = v
    return ops


def brickwork_ops(n, depth, seed, uniforms):
    """The random U + CX brick wall as flat ops, for harnesses that drive ket
    without the B200 package.  Every layer applies U(theta, phi, lambda) to
    every qubit (angles uniform on [0, 2pi), three draws per qubit in (layer,
    qubit, theta/phi/lambda) order from std::mt19937{seed}), then CX on pairs
    (a, a+1) for a = layer mod 2, layer mod 2 + 2, ...  `uniforms(seed,
    count)` supplies uniform_real_distribution<double>(0, 1) draws; scaling
    by 2pi is exact for libstdc++'s (b - a) * u + a with a = 0."""
    two_pi = 6.283185307179586
    u = uniforms(seed, 3 * n * depth) * two_pi
    gates = []
    k = 0
    for layer in range(depth):
        for q in range(n):
            gates.append(("U", (q,), (u[k], u[k + 1], u[k + 2])))
            k += 3
        for a in range(layer % 2, n - 1, 2):
            gates.append(("CX", (a, a + 1)))
    return make_ops(gates)


def build_oracle():
    """Compile the C restatement (fast; gcc only)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def _ptr(a, t=ct.c_double):
    return a.ctypes.data_as(ct.POINTER(t))


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build_oracle()
        L = ct.CDLL(path)
        vp, sz, i32 = ct.c_void_p, ct.c_size_t, ct.c_int
        L.ko_apply.argtypes = [i32, vp, vp, sz, i32]
        L.ko_run.argtypes = [i32, vp, sz, i32, vp]
        L.ko_apply_matrix.argtypes = [i32, vp, vp, i32, vp]
        L.ko_block_matrix.argtypes = [vp, sz, vp, i32, vp]
        L.ko_expval.argtypes = [i32, vp, ct.c_char_p, ct.POINTER(i32)]
        L.ko_expval.restype = ct.c_double
        L.ko_expval_sum.argtypes = [i32, vp, vp, vp, sz, ct.POINTER(i32)]
        L.ko_expval_sum.restype = ct.c_double
        L.ko_measure_sequential.argtypes = [i32, vp, ct.c_double]
        L.ko_measure_sequential.restype = ct.c_uint64
        L.ko_measure_sequential_many.argtypes = [i32, vp, vp, sz, vp]
        L.ko_measure_sequential_many32.argtypes = [i32, vp, vp, sz, vp]
        L.ko_uniforms_mt19937.argtypes = [ct.c_uint32, sz, vp]
        L.ko_sample_tree.argtypes = [i32, vp, vp, vp, sz, vp]
        L.ko_adjoint.argtypes = [i32, vp, sz, vp, vp, sz, vp, vp, sz, vp, vp]
        L.ko_mlp_forward.argtypes = [vp] * 7 + [i32, vp]
        L.ko_mlp_backward.argtypes = [vp] * 8 + [i32] + [vp] * 6
        L.ko_mlp_backward.restype = ct.c_double
        self.L = L

    # ket::run restated; fuse=1 follows ket's Fuser exactly.
    def run(self, n, ops, fuse=1):
        amps = np.zeros(2 << n, dtype=np.float64)
        rc = self.L.ko_run(n, ops.ctypes.data, len(ops), fuse, amps.ctypes.data)
        if rc != 0:
            raise ValueError("oracle: malformed op")
        return amps.view(np.complex128)

    def apply(self, n, state, ops, fuse=1):
        st = np.ascontiguousarray(state, dtype=np.complex128).copy()
        rc = self.L.ko_apply(n, st.ctypes.data, ops.ctypes.data, len(ops), fuse)
        if rc != 0:
            raise ValueError("oracle: malformed op")
        return st

    def apply_matrix(self, n, state, qubits, mat):
        st = np.ascontiguousarray(state, dtype=np.complex128).copy()
        q = np.asarray(qubits, dtype=np.int32)
        m = np.ascontiguousarray(mat, dtype=np.complex128)
        self.L.ko_apply_matrix(n, st.ctypes.data, q.ctypes.data, len(q), m.ctypes.data)
        return st

    def block_matrix(self, ops, qubits):
        q = np.asarray(qubits, dtype=np.int32)
        d = 1 << len(q)
        m = np.zeros((d, d), dtype=np.complex128)
        if self.L.ko_block_matrix(ops.ctypes.data, len(ops), q.ctypes.data, len(q), m.ctypes.data):
            raise ValueError("oracle: gate outside block")
        return m

    def expval(self, n, state, pauli):
        st = np.ascontiguousarray(state, dtype=np.complex128)
        err = ct.c_int(0)
        v = self.L.ko_expval(n, st.ctypes.data, pauli.encode(), ct.byref(err))
        if err.value:
            raise ValueError({-1: "size", -2: "length", -3: "character"}[err.value])
        return v

    def expval_sum(self, n, state, terms):
        st = np.ascontiguousarray(state, dtype=np.complex128)
        coeffs = np.array([c for c, _ in terms], dtype=np.float64)
        bufs = [ct.create_string_buffer(p.encode()) for _, p in terms]
        arr = (ct.c_char_p * len(terms))(*[ct.cast(b, ct.c_char_p) for b in bufs])
        err = ct.c_int(0)
        v = self.L.ko_expval_sum(n, st.ctypes.data, coeffs.ctypes.data,
                                 ct.cast(arr, ct.c_void_p), len(terms), ct.byref(err))
        if err.value:
            raise ValueError("bad pauli")
        return v

    def uniforms(self, seed, count):
        out = np.zeros(count, dtype=np.float64)
        self.L.ko_uniforms_mt19937(seed, count, out.ctypes.data)
        return out

    def measure_sequential(self, n, state, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.zeros(len(u), dtype=np.uint64)
        if state.dtype == np.complex64:
            st = np.ascontiguousarray(state)
            self.L.ko_measure_sequential_many32(n, st.ctypes.data, u.ctypes.data, len(u), out.ctypes.data)
        else:
            st = np.ascontiguousarray(state, dtype=np.complex128)
            self.L.ko_measure_sequential_many(n, st.ctypes.data, u.ctypes.data, len(u), out.ctypes.data)
        return out

    def sample_tree(self, n, state, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.zeros(len(u), dtype=np.uint64)
        if state.dtype == np.complex64:
            st = np.ascontiguousarray(state)
            self.L.ko_sample_tree(n, None, st.ctypes.data, u.ctypes.data, len(u), out.ctypes.data)
        else:
            st = np.ascontiguousarray(state, dtype=np.complex128)
            self.L.ko_sample_tree(n, st.ctypes.data, None, u.ctypes.data, len(u), out.ctypes.data)
        return out

    def adjoint(self, n, ops, param_index, params, terms):
        pidx = np.ascontiguousarray(param_index, dtype=np.int32)
        prm = np.ascontiguousarray(params, dtype=np.float64)
        coeffs = np.array([c for c, _ in terms], dtype=np.float64)
        bufs = [ct.create_string_buffer(p.encode()) for _, p in terms]
        arr = (ct.c_char_p * len(terms))(*[ct.cast(b, ct.c_char_p) for b in bufs])
        grad = np.zeros(len(prm), dtype=np.float64)
        val = np.zeros(1, dtype=np.float64)
        rc = self.L.ko_adjoint(n, ops.ctypes.data, len(ops), pidx.ctypes.data, prm.ctypes.data,
                               len(prm), coeffs.ctypes.data, ct.cast(arr, ct.c_void_p),
                               len(terms), val.ctypes.data, grad.ctypes.data)
        if rc:
            raise ValueError("oracle adjoint failed: %d" % rc)
        return float(val[0]), grad

    def mlp_forward(self, w, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.zeros(x.shape[0], dtype=np.float64)
        ws = [np.ascontiguousarray(a, dtype=np.float32) for a in w]
        self.L.ko_mlp_forward(*[a.ctypes.data for a in ws], x.ctypes.data, x.shape[0], out.ctypes.data)
        return out

    def mlp_backward(self, w, x, y):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        ws = [np.ascontiguousarray(a, dtype=np.float32) for a in w]
        grads = [np.zeros(a.shape, dtype=np.float64) for a in ws]
        loss = self.L.ko_mlp_backward(*[a.ctypes.data for a in ws], x.ctypes.data, y.ctypes.data,
                                      x.shape[0], *[g.ctypes.data for g in grads])
        return loss, grads


class Reference:
    """ket itself (or the drop-in build) through ref_shim.cpp."""

    def __init__(self, dropin: bool = False):
        path = DROPIN_SO if dropin else REF_SO
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = ct.CDLL(path)
        vp, sz, i32, u32 = ct.c_void_p, ct.c_size_t, ct.c_int, ct.c_uint32
        L.ref_last_error.restype = ct.c_char_p
        L.ref_set_num_threads.argtypes = [ct.c_uint]
        L.ref_num_threads.restype = ct.c_uint
        L.ref_run.argtypes = [i32, vp, sz, vp]
        L.ref_run_timed.argtypes = [i32, vp, sz, vp, vp]
        if hasattr(L, "ref_run_timed_state"):
            L.ref_run_timed_state.argtypes = [i32, vp, sz, vp, vp]
        L.ref_run_with_probes.argtypes = [i32, vp, sz, vp, vp, sz, vp]
        L.ref_expval.argtypes = [i32, vp, ct.c_char_p, vp]
        L.ref_expval_sum.argtypes = [i32, vp, vp, vp, sz, vp]
        L.ref_expval_circuit.argtypes = [i32, vp, sz, vp, vp, sz, i32, vp]
        L.ref_measure.argtypes = [i32, vp, u32, sz, vp]
        L.ref_uniforms.argtypes = [u32, sz, vp]
        L.ref_sample.argtypes = [i32, vp, sz, u32, i32, sz, vp, vp]
        L.ref_simulate_sample.argtypes = [i32, vp, sz, u32, i32, sz, vp, vp, ct.c_char_p, sz]
        L.ref_is_clifford.argtypes = [i32, vp, sz, vp]
        L.ref_chosen_method.argtypes = [i32, vp, sz, vp]
        for name in ("ref_qasm_parse", "ref_qasm_roundtrip", "ref_to_qasm", "ref_state_print",
                     "ref_stepper_walk", "ref_stepper_seek"):
            if not hasattr(L, name):  # built before the OpenQASM entry points
                break
        else:
            L.ref_qasm_parse.argtypes = [ct.c_char_p, vp, vp, vp, vp, sz, vp]
            L.ref_qasm_roundtrip.argtypes = [ct.c_char_p, vp, sz, vp]
            L.ref_to_qasm.argtypes = [i32, vp, sz, vp, sz, vp]
            L.ref_state_print.argtypes = [i32, vp, vp, sz, vp]
            L.ref_stepper_walk.argtypes = [i32, vp, sz, vp, sz, vp]
            L.ref_stepper_seek.argtypes = [i32, vp, sz, vp, sz, vp, vp]
        self.L = L

    def _check(self, rc):
        if rc == 0:
            return
        msg = self.L.ref_last_error().decode()
        raise {-1: IndexError, -2: ValueError}.get(rc, RuntimeError)(msg)

    def set_num_threads(self, t):
        self.L.ref_set_num_threads(t)

    def num_threads(self):
        return self.L.ref_num_threads()

    def run(self, n, ops):
        amps = np.zeros(2 << n, dtype=np.float64)
        self._check(self.L.ref_run(n, ops.ctypes.data, len(ops), amps.ctypes.data))
        return amps.view(np.complex128)

    def run_timed_state(self, n, ops):
        """(seconds of ket::run alone, the state it returned)."""
        secs = np.zeros(1)
        amps = np.empty(2 << n, dtype=np.float64)
        self._check(self.L.ref_run_timed_state(n, ops.ctypes.data, len(ops), secs.ctypes.data,
                                               amps.ctypes.data))
        return float(secs[0]), amps.view(np.complex128)

    def run_timed(self, n, ops):
        secs = np.zeros(1)
        a0 = np.zeros(2)
        self._check(self.L.ref_run_timed(n, ops.ctypes.data, len(ops), secs.ctypes.data, a0.ctypes.data))
        return float(secs[0])

    def run_with_probes(self, n, ops, max_probes=16):
        dim = 1 << n
        final = np.zeros(2 * dim)
        probes = np.zeros(2 * dim * max_probes)
        cnt = ct.c_size_t(0)
        self._check(self.L.ref_run_with_probes(n, ops.ctypes.data, len(ops), final.ctypes.data,
                                               probes.ctypes.data, max_probes, ct.byref(cnt)))
        k = min(cnt.value, max_probes)
        return final.view(np.complex128), probes.view(np.complex128).reshape(max_probes, dim)[:k]

    def expval(self, n, state, pauli):
        st = np.ascontiguousarray(state, dtype=np.complex128)
        out = np.zeros(1)
        self._check(self.L.ref_expval(n, st.ctypes.data, pauli.encode(), out.ctypes.data))
        return float(out[0])

    def expval_sum(self, n, state, terms):
        st = np.ascontiguousarray(state, dtype=np.complex128)
        coeffs = np.array([c for c, _ in terms], dtype=np.float64)
        bufs = [ct.create_string_buffer(p.encode()) for _, p in terms]
        arr = (ct.c_char_p * len(terms))(*[ct.cast(b, ct.c_char_p) for b in bufs])
        out = np.zeros(1)
        self._check(self.L.ref_expval_sum(n, st.ctypes.data, coeffs.ctypes.data,
                                          ct.cast(arr, ct.c_void_p), len(terms), out.ctypes.data))
        return float(out[0])

    def expval_circuit(self, n, ops, terms, method=0):
        coeffs = np.array([c for c, _ in terms], dtype=np.float64)
        bufs = [ct.create_string_buffer(p.encode()) for _, p in terms]
        arr = (ct.c_char_p * len(terms))(*[ct.cast(b, ct.c_char_p) for b in bufs])
        out = np.zeros(1)
        self._check(self.L.ref_expval_circuit(n, ops.ctypes.data, len(ops), coeffs.ctypes.data,
                                              ct.cast(arr, ct.c_void_p), len(terms), method,
                                              out.ctypes.data))
        return float(out[0])

    def measure(self, n, state, seed, shots):
        st = np.ascontiguousarray(state, dtype=np.complex128)
        out = np.zeros(shots, dtype=np.uint64)
        self._check(self.L.ref_measure(n, st.ctypes.data, seed, shots, out.ctypes.data))
        return out

    def uniforms(self, seed, count):
        out = np.zeros(count, dtype=np.float64)
        self.L.ref_uniforms(seed, count, out.ctypes.data)
        return out

    def sample(self, n, ops, seed, shots, method=0, evolve_once=False):
        ncl = int(max([o["q"][1] + 1 for o in ops if o["type"] == CODE["Measure"]] or [0]))
        creg = np.zeros(max(1, shots * ncl), dtype=np.int32)
        cnt = ct.c_size_t(0)
        if evolve_once:
            name = ct.create_string_buffer(64)
            self._check(self.L.ref_simulate_sample(n, ops.ctypes.data, len(ops), seed, method, shots,
                                                   creg.ctypes.data, ct.byref(cnt), name, 64))
            return creg[: shots * cnt.value].reshape(shots, cnt.value), name.value.decode()
        self._check(self.L.ref_sample(n, ops.ctypes.data, len(ops), seed, method, shots,
                                      creg.ctypes.data, ct.byref(cnt)))
        return creg[: shots * cnt.value].reshape(shots, cnt.value)

    def is_clifford(self, n, ops):
        out = ct.c_int(0)
        self._check(self.L.ref_is_clifford(n, ops.ctypes.data, len(ops), ct.byref(out)))
        return bool(out.value)

    def chosen_method(self, n, ops):
        out = ct.c_int(0)
        self._check(self.L.ref_chosen_method(n, ops.ctypes.data, len(ops), ct.byref(out)))
        return "stabilizer" if out.value == 2 else "statevector"

    # -- OpenQASM (bindings/qasm/qasm.cpp) -----------------------------------
    def qasm_parse(self, src):
        """ket::from_qasm: register sizes, top-level node count and the gates
        with composites expanded (barriers keep their width in nq)."""
        nq, nc, top, n = ct.c_int(), ct.c_int(), ct.c_int(), ct.c_size_t()
        ops = np.zeros(4096, dtype=OP_DTYPE)
        b = src.encode()
        self._check(self.L.ref_qasm_parse(b, ct.byref(nq), ct.byref(nc), ct.byref(top), ops.ctypes.data,
                                          len(ops), ct.byref(n)))
        if n.value > len(ops):
            ops = np.zeros(n.value, dtype=OP_DTYPE)
            self._check(self.L.ref_qasm_parse(b, ct.byref(nq), ct.byref(nc), ct.byref(top), ops.ctypes.data,
                                              len(ops), ct.byref(n)))
        return {"n_qubits": nq.value, "n_clbits": nc.value, "n_top": top.value, "ops": ops[:n.value].copy()}

    def _text(self, call):
        size = ct.c_size_t()
        buf = ct.create_string_buffer(1 << 16)
        self._check(call(buf, len(buf), ct.byref(size)))
        if size.value >= len(buf):
            buf = ct.create_string_buffer(size.value + 1)
            self._check(call(buf, len(buf), ct.byref(size)))
        return buf.raw[:size.value].decode()

    def qasm_roundtrip(self, src):
        """ket::to_qasm(ket::from_qasm(src))."""
        b = src.encode()
        return self._text(lambda buf, cap, n: self.L.ref_qasm_roundtrip(b, buf, cap, n))

    def to_qasm(self, n, ops):
        """ket::to_qasm of a circuit built from flat ops."""
        return self._text(lambda buf, cap, k: self.L.ref_to_qasm(n, ops.ctypes.data, len(ops), buf, cap, k))

    def state_print(self, n, state):
        """ket::State::print of 2^n complex amplitudes."""
        a = np.ascontiguousarray(state, dtype=np.complex128)
        return self._text(lambda buf, cap, k: self.L.ref_state_print(n, a.ctypes.data, buf, cap, k))

    # -- Stepper (include/ket/stepper.hpp) ------------------------------------
    def stepper_walk(self, n, ops):
        """States at every position of ket::Stepper stepped to the end."""
        cap = len(ops) + 1
        out = np.zeros((cap, 1 << n), dtype=np.complex128)
        steps = ct.c_size_t()
        self._check(self.L.ref_stepper_walk(n, ops.ctypes.data, len(ops), out.ctypes.data, cap, ct.byref(steps)))
        return out[:steps.value + 1]

    def stepper_seek(self, n, ops, seq):
        """ket::Stepper::seek(k) for each k of seq: (states, positions)."""
        seq = np.ascontiguousarray(seq, dtype=np.uint64)
        out = np.zeros((len(seq), 1 << n), dtype=np.complex128)
        pos = np.zeros(len(seq), dtype=np.uint64)
        self._check(self.L.ref_stepper_seek(n, ops.ctypes.data, len(ops), seq.ctypes.data, len(seq),
                                            out.ctypes.data, pos.ctypes.data))
        return out, pos
