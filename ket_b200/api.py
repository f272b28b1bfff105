"""ket's Python API on the B200 backend (bindings/python/module.cpp:41-271).

Same names and argument meaning as ket's ``_ket`` module -- ``run``,
``run_with_probes``, ``expval`` (four overloads), ``measure``, ``sample``,
``is_clifford``, ``chosen_method``, ``set_num_threads``/``num_threads`` --
with every state-vector computation on the GPU through the C ABI.  Extras
for large states: ``run_device`` returns a ``DeviceState`` that never leaves
HBM, and ``set_options`` selects precision (complex128 by default, as ket),
fusion mode and the tensor-core path.
"""
from __future__ import annotations

import ctypes as ct
import math
import os
import threading
from typing import Iterable, List, Optional, Sequence, Tuple, Union

import numpy as np

from . import _lib
from ._lib import C64, C128, FUSE_GREEDY, FUSE_LEARNED, FUSE_NONE, FUSE_REFERENCE, check, lib
from .circuit import Circuit

_PRECISIONS = {"c64": C64, "complex64": C64, "c128": C128, "complex128": C128}
_FUSIONS = {"none": FUSE_NONE, "unfused": FUSE_NONE, "reference": FUSE_REFERENCE,
            "greedy": FUSE_GREEDY, "learned": FUSE_LEARNED}

_opts = _lib.Options(C128, FUSE_GREEDY, 0, 1, 0)
_num_threads = [1]


def set_options(precision=None, fusion=None, max_block_qubits=None, tensor_cores=None):
    """Backend options for later ``run``/``sample``/``expval`` calls."""
    if precision is not None:
        _opts.precision = _PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    if fusion is not None:
        _opts.fusion = _FUSIONS[fusion] if isinstance(fusion, str) else int(fusion)
        if _opts.fusion == FUSE_LEARNED:
            use_learned_planner()
    if max_block_qubits is not None:
        _opts.max_block_qubits = int(max_block_qubits)
    if tensor_cores is not None:
        _opts.tensor_cores = 1 if tensor_cores else 0


_model = [None]


def use_learned_planner(path: Optional[str] = None):
    """Attach the trained cost model (ket_b200/data/cost_model.npz unless
    `path` is given) to the planner's FUSE_LEARNED mode; returns it."""
    from .planner import DEFAULT_MODEL, CostModel
    if _model[0] is None or path is not None:
        m = CostModel.load(path or DEFAULT_MODEL)
        m.attach()
        _model[0] = m
    return _model[0]


def get_options() -> dict:
    inv_p = {C64: "c64", C128: "c128"}
    inv_f = {FUSE_NONE: "none", FUSE_REFERENCE: "reference", FUSE_GREEDY: "greedy", FUSE_LEARNED: "learned"}
    return {"precision": inv_p[_opts.precision], "fusion": inv_f[_opts.fusion],
            "max_block_qubits": _opts.max_block_qubits, "tensor_cores": bool(_opts.tensor_cores)}


def make_options(precision="c128", fusion="greedy", max_block_qubits=0, tensor_cores=True,
                 renormalize=0) -> _lib.Options:
    """max_block_qubits 0 takes the library default (6 for complex64 on the
    tensor cores, else 5); renormalize: 0 restores the starting norm after
    tensor-core blocks, -1 never, 1 after every plan."""
    return _lib.Options(_PRECISIONS[precision] if isinstance(precision, str) else int(precision),
                        _FUSIONS[fusion] if isinstance(fusion, str) else int(fusion),
                        int(max_block_qubits), 1 if tensor_cores else 0, int(renormalize))


def set_num_threads(threads: int) -> None:
    """Accepted for ket compatibility (parallelism.hpp:17); the GPU path
    sizes its own grids, so the value only changes ``num_threads()``."""
    if threads < 0:
        raise ValueError("threads must be non-negative")
    _num_threads[0] = threads if threads else (os.cpu_count() or 1)


def num_threads() -> int:
    return _num_threads[0]


# ---------------------------------------------------------------------------
class DeviceState:
    """A 2^n state vector resident in GPU memory (complex64 or complex128)."""

    def __init__(self, n_qubits: int, precision="c128"):
        p = _PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        h = ct.c_void_p()
        check(lib.ketgpu_state_create(int(n_qubits), p, ct.byref(h)))
        self._h = h
        self.n_qubits = int(n_qubits)
        self.precision = p

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib.ketgpu_state_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return 1 << self.n_qubits

    def reset(self):
        check(lib.ketgpu_state_reset(self._h))

    def apply(self, circuit: Union[Circuit, np.ndarray], options: Optional[_lib.Options] = None):
        ops = circuit.to_ops() if isinstance(circuit, Circuit) else np.ascontiguousarray(circuit)
        opt = options or _lib.Options(self.precision, _opts.fusion, _opts.max_block_qubits, _opts.tensor_cores, 0)
        check(lib.ketgpu_apply(self._h, ops.ctypes.data, len(ops), ct.byref(opt)))
        return self

    def to_numpy(self, first: int = 0, count: Optional[int] = None) -> np.ndarray:
        dim = 1 << self.n_qubits
        count = dim - first if count is None else count
        out = np.empty(count, dtype=np.complex128)
        check(lib.ketgpu_state_download(self._h, first, count, out.ctypes.data))
        return out

    def to_numpy_raw(self, first: int = 0, count: Optional[int] = None) -> np.ndarray:
        """Amplitudes in the state's own precision (complex64 or complex128)."""
        dim = 1 << self.n_qubits
        count = dim - first if count is None else count
        out = np.empty(count, dtype=np.complex64 if self.precision == C64 else np.complex128)
        check(lib.ketgpu_state_download_raw(self._h, first, count, out.ctypes.data))
        return out

    def from_numpy(self, amps: np.ndarray, first: int = 0):
        a = np.ascontiguousarray(amps, dtype=np.complex128)
        check(lib.ketgpu_state_upload(self._h, first, len(a), a.ctypes.data))
        return self

    def __getitem__(self, i: int) -> complex:
        if not (0 <= i < len(self)):
            raise IndexError()
        return complex(self.to_numpy(i, 1)[0])

    def norm(self) -> float:
        v = ct.c_double()
        check(lib.ketgpu_norm(self._h, ct.byref(v)))
        return v.value

    def inner(self, other: "DeviceState") -> complex:
        re, im = ct.c_double(), ct.c_double()
        check(lib.ketgpu_inner(self._h, other._h, ct.byref(re), ct.byref(im)))
        return complex(re.value, im.value)

    def compare(self, other: "DeviceState") -> dict:
        """max |a-b|, fidelity |<a|b>|^2/(<a|a><b|b>), overlap and norms (any precisions)."""
        out = np.zeros(5)
        check(lib.ketgpu_compare(self._h, other._h, out.ctypes.data))
        ov = complex(out[1], out[2])
        return {"max_abs": float(out[0]), "overlap": ov, "norm_a": float(out[3]), "norm_b": float(out[4]),
                "fidelity": abs(ov) ** 2 / (out[3] * out[4]) if out[3] > 0 and out[4] > 0 else 0.0,
                "fidelity_unnormalised": abs(ov) ** 2}

    def expval(self, obs) -> float:
        return _expval_dev(self, obs)

    def sample(self, uniforms: np.ndarray) -> np.ndarray:
        u = np.ascontiguousarray(uniforms, dtype=np.float64)
        out = np.empty(len(u), dtype=np.uint64)
        check(lib.ketgpu_sample(self._h, u.ctypes.data, len(u), out.ctypes.data))
        return out

    def sample_seeded(self, seed: int, count: int) -> np.ndarray:
        """`count` draws with the uniforms of std::mt19937{seed}, in order
        (ketgpu_sample_seeded); the sampling tree is reused while the state
        is unchanged."""
        out = np.empty(count, dtype=np.uint64)
        check(lib.ketgpu_sample_seeded(self._h, int(seed) & 0xFFFFFFFF, count, out.ctypes.data))
        return out

    def torch_view(self):
        """Zero-copy torch tensor over the device amplitudes (complex)."""
        import torch
        ptr = lib.ketgpu_state_device_ptr(self._h)
        n = 1 << self.n_qubits
        dt = torch.complex64 if self.precision == C64 else torch.complex128

        class _CAI:
            __cuda_array_interface__ = {
                "shape": (n,), "typestr": "<c8" if self.precision == C64 else "<c16",
                "data": (ptr, False), "version": 3, "strides": None}
        return torch.as_tensor(_CAI(), device="cuda").view(dt)


def _num_text(x: float) -> str:
    if math.isnan(x):  # C's printf shows the sign of a NaN
        return "-nan" if math.copysign(1.0, x) < 0 else "nan"
    return "%g" % x


def _amp_text(z: complex) -> str:
    """An amplitude as ket writes it (src/state.cpp:20-32)."""
    re_, im = z.real, z.imag
    if im == 0.0:
        return _num_text(re_)
    if re_ == 0.0:
        return _num_text(im) + "i"
    if im < 0.0:
        return f"{_num_text(re_)} - {_num_text(-im)}i"
    return f"{_num_text(re_)} + {_num_text(im)}i"


class State:
    """ket.State: 2^n complex128 amplitudes on the host (state.hpp:15-34),
    keeping the device copy it was produced from for further queries."""

    def __init__(self, amps: np.ndarray, device: Optional[DeviceState] = None):
        self._amps = np.ascontiguousarray(amps, dtype=np.complex128)
        self._dev = device

    def __len__(self):
        return len(self._amps)

    def __getitem__(self, i: int) -> complex:
        if not (0 <= i < len(self._amps)):
            raise IndexError()
        return complex(self._amps[i])

    def __repr__(self):
        return f"<ket_b200.State size={len(self._amps)}>"

    def print(self) -> str:
        """ket.State.print (src/state.cpp:42-52): one line per amplitude,
        ``|b_{n-1}...b_0⟩: amplitude``, numbers as C++ streams write a double
        by default (6 significant digits)."""
        n = 0
        while (1 << n) < len(self._amps):
            n += 1
        return "".join(f"|{format(i, f'0{n}b') if n else ''}⟩: {_amp_text(z)}\n"
                       for i, z in enumerate(self._amps.tolist()))

    __str__ = print

    def to_numpy(self) -> np.ndarray:
        return self._amps

    @property
    def n_qubits(self) -> int:
        return int(len(self._amps)).bit_length() - 1

    def device(self) -> DeviceState:
        if self._dev is None:
            d = DeviceState(self.n_qubits, C128)
            d.from_numpy(self._amps)
            self._dev = d
        return self._dev


class ProbeRun:
    def __init__(self, final: State, probes: List[Tuple[str, State]]):
        self.final = final
        self.probes = probes


# ---------------------------------------------------------------------------
def run_device(circuit: Circuit, precision=None, options: Optional[_lib.Options] = None) -> DeviceState:
    """Evolve |0...0> on the GPU and keep the state there."""
    opt = options or _lib.Options(_opts.precision, _opts.fusion, _opts.max_block_qubits, _opts.tensor_cores, 0)
    if precision is not None:
        opt.precision = _PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    d = DeviceState(circuit.n_qubits, opt.precision)
    d.apply(circuit, opt)
    return d


def run(circuit: Circuit) -> State:
    """ket.run (simulator.hpp:15): the final state as a host State."""
    d = run_device(circuit)
    return State(d.to_numpy(), d)


def run_with_probes(circuit: Circuit) -> ProbeRun:
    """ket.run_with_probes (simulator.hpp:24, simulator.cpp:560-565)."""
    from .circuit import GateType
    d = DeviceState(circuit.n_qubits, _opts.precision)
    probes = []
    segment = Circuit(circuit.n_qubits)
    for g in circuit.flat_gates():
        if g.type == GateType.Probe:
            d.apply(segment)
            probes.append((g.label, State(d.to_numpy())))
            segment = Circuit(circuit.n_qubits)
        else:
            segment._gates.append(g)
    d.apply(segment)
    return ProbeRun(State(d.to_numpy(), d), probes)


def _terms(obs) -> List[Tuple[float, str]]:
    if isinstance(obs, str):
        return [(1.0, obs)]
    return [(float(c), str(p)) for c, p in obs]


def _expval_dev(d: DeviceState, obs) -> float:
    if isinstance(obs, str):
        out = ct.c_double()
        check(lib.ketgpu_expval(d.handle, obs.encode(), ct.byref(out)))
        return out.value
    terms = _terms(obs)
    coeffs = np.array([c for c, _ in terms], dtype=np.float64)
    arr, keep = _lib.c_strings([p for _, p in terms])
    out = ct.c_double()
    check(lib.ketgpu_expval_sum(d.handle, coeffs.ctypes.data, ct.cast(arr, ct.c_void_p), len(terms),
                                ct.byref(out)))
    return out.value


def _method(method: str) -> str:
    if method not in ("auto", "statevector", "stabilizer"):
        raise ValueError("method must be 'auto', 'statevector', or 'stabilizer'")
    return method


def is_clifford(circuit: Circuit) -> bool:
    return circuit.is_clifford()


def chosen_method(circuit: Circuit) -> str:
    return "stabilizer" if circuit.is_clifford() else "statevector"


def _resolve(circuit: Circuit, method: str) -> str:
    method = _method(method)
    if method == "auto":
        method = chosen_method(circuit)
    if method == "stabilizer" and not circuit.is_clifford():
        raise ValueError("stabilizer backend requires a Clifford circuit (it contains a non-Clifford gate); "
                         "use Method::Auto or Method::StateVector")
    return method


def _stabilizer():
    """ket's own CPU stabilizer tableau (src/backends/stabilizer.cpp), which
    this backend leaves untouched: ket's Python module when it is installed."""
    try:
        import ket as _ket  # the reference package
        return _ket
    except ImportError as e:
        raise RuntimeError(
            "Clifford circuits are simulated by ket's own stabilizer tableau; install ket "
            "(or link the C++ drop-in into ket) to use method='stabilizer'") from e


def _to_ket(circuit: Circuit):
    k = _stabilizer()
    c = k.Circuit(circuit.n_qubits)
    from .circuit import GateType as G
    for g in circuit.flat_gates():
        name = {G.H: "h", G.X: "x", G.Y: "y", G.Z: "z", G.S: "s", G.Sdg: "sdg", G.CX: "cx",
                G.CY: "cy", G.CZ: "cz", G.Swap: "swap"}.get(g.type)
        if name:
            getattr(c, name)(*g.qubits)
        elif g.type == G.Measure:
            c.measure(g.qubits[0], g.clbit)
        elif g.type == G.Barrier:
            c.barrier()
    return c


def expval(target, obs, method: str = "auto") -> float:
    """The four overloads of ket.expval (module.cpp:180-213)."""
    if isinstance(target, State):
        return _expval_dev(target.device(), obs)
    if isinstance(target, DeviceState):
        return _expval_dev(target, obs)
    if isinstance(target, Circuit):
        m = _resolve(target, method)
        if m == "stabilizer":
            k = _stabilizer()
            return k.expval(_to_ket(target), obs if isinstance(obs, str) else list(obs), "stabilizer")
        d = run_device(target)
        try:
            return _expval_dev(d, obs)
        finally:
            d.close()
    raise TypeError("expval: expected a State, DeviceState or Circuit")


_tls = threading.local()


def _auto_seed() -> int:
    return int.from_bytes(os.urandom(4), "little")


def uniforms(seed: int, count: int) -> np.ndarray:
    """The draws of uniform_real_distribution<double>(0,1) on std::mt19937{seed}."""
    out = np.empty(count, dtype=np.float64)
    check(lib.ketgpu_uniforms_mt19937(int(seed) & 0xFFFFFFFF, count, out.ctypes.data))
    return out


def measure(state, seed: Optional[int] = None) -> int:
    """ket.measure (module.cpp:242-253): one Born-rule draw."""
    d = state.device() if isinstance(state, State) else state
    out = ct.c_uint64()
    check(lib.ketgpu_measure(d.handle, (_auto_seed() if seed is None else int(seed)) & 0xFFFFFFFF,
                             ct.byref(out)))
    return int(out.value)


def sample(circuit: Circuit, seed: Optional[int] = None, method: str = "auto") -> List[int]:
    """ket.sample (module.cpp:255-270): one shot of the circuit's measurements."""
    m = _resolve(circuit, method)
    if m == "stabilizer":
        k = _stabilizer()
        return list(k.sample(_to_ket(circuit), seed, "stabilizer"))
    d = run_device(circuit)
    try:
        u = uniforms(_auto_seed() if seed is None else int(seed), 1)
        outcome = int(d.sample(u)[0])
    finally:
        d.close()
    creg = [0] * circuit.n_clbits
    for q, cb in circuit.measurements():
        creg[cb] = (outcome >> q) & 1
    return creg


def sample_shots(circuit: Circuit, shots: int, seed: int = 0) -> np.ndarray:
    """Many shots from one evolution (one CDF), the draws of one
    std::mt19937{seed} stream in order; returns shots x n_clbits."""
    d = run_device(circuit)
    try:
        outcomes = d.sample_seeded(seed, shots)
    finally:
        d.close()
    meas = circuit.measurements()
    creg = np.zeros((shots, circuit.n_clbits), dtype=np.int32)
    for q, cb in meas:
        creg[:, cb] = ((outcomes >> np.uint64(q)) & np.uint64(1)).astype(np.int32)
    return creg


def plan_stats(circuit: Circuit, options: Optional[_lib.Options] = None) -> dict:
    ops = circuit.to_ops()
    opt = options or _lib.Options(_opts.precision, _opts.fusion, _opts.max_block_qubits, _opts.tensor_cores, 0)
    h = ct.c_void_p()
    check(lib.ketgpu_plan_create(circuit.n_qubits, ops.ctypes.data, len(ops), ct.byref(opt), ct.byref(h)))
    st = _lib.PlanStats()
    try:
        check(lib.ketgpu_plan_stats_get(h, ct.byref(st)))
    finally:
        lib.ketgpu_plan_destroy(h)
    return {f: getattr(st, f) for f, _ in _lib.PlanStats._fields_}


class Plan:
    """A compiled circuit (fusion blocks, matrices on the device) for repeated runs."""

    def __init__(self, n_qubits: int, ops: np.ndarray, options: _lib.Options):
        self.n_qubits = n_qubits
        self._ops = np.ascontiguousarray(ops)
        h = ct.c_void_p()
        check(lib.ketgpu_plan_create(n_qubits, self._ops.ctypes.data, len(self._ops), ct.byref(options),
                                     ct.byref(h)))
        self._h = h

    def stats(self) -> dict:
        st = _lib.PlanStats()
        check(lib.ketgpu_plan_stats_get(self._h, ct.byref(st)))
        return {f: getattr(st, f) for f, _ in _lib.PlanStats._fields_}

    def pass_info(self, index: int) -> dict:
        """Kind (0 pair, 1 phase, 2 dense block, 3 norm, 4 diagonal run),
        qubits k, tensor-core flag and algorithmic HBM bytes of one pass."""
        kind, k, tc, b = ct.c_int32(), ct.c_int32(), ct.c_int32(), ct.c_double()
        check(lib.ketgpu_plan_pass_info(self._h, index, ct.byref(kind), ct.byref(k), ct.byref(tc), ct.byref(b)))
        return {"kind": kind.value, "k": k.value, "tensor": bool(tc.value), "bytes": b.value}

    def pass_qubits(self, index: int) -> List[int]:
        """The qubits one pass acts on, ascending (dense block: matrix bit b is
        qubits[b]); empty for norm passes and diagonal runs."""
        buf = (ct.c_int32 * 8)()
        cnt = ct.c_int32()
        check(lib.ketgpu_plan_pass_qubits(self._h, index, buf, 8, ct.byref(cnt)))
        return [buf[i] for i in range(min(cnt.value, 8))]

    def pass_gates(self, index: int) -> List[int]:
        """Indices of the ops pass `index` applies, in its order."""
        cnt = ct.c_int32()
        check(lib.ketgpu_plan_pass_gates(self._h, index, None, 0, ct.byref(cnt)))
        buf = (ct.c_int32 * max(1, cnt.value))()
        check(lib.ketgpu_plan_pass_gates(self._h, index, buf, cnt.value, ct.byref(cnt)))
        return list(buf[:cnt.value])

    def pass_tc_form(self, index: int) -> dict:
        """How a tensor-core pass runs: ``tma_dims`` (dimensions of the
        tensor map fetching each tile; 0 = per-thread cp.async) and
        ``direct`` (epilogue stores straight from registers)."""
        t, d = ct.c_int32(), ct.c_int32()
        check(lib.ketgpu_plan_pass_tc_form(self._h, index, ct.byref(t), ct.byref(d)))
        return {"tma_dims": t.value, "direct": bool(d.value)}

    def pass_bytes(self, index: int) -> float:
        return self.pass_info(index)["bytes"]

    def execute(self, state: DeviceState, sync: bool = True):
        check(lib.ketgpu_plan_execute(self._h, state.handle))
        if sync:
            check(lib.ketgpu_state_synchronize(state.handle))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib.ketgpu_plan_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
