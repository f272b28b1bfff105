"""Circuit recorder with ket's builder API (include/ket/circuit.hpp:16-162).

A ``Circuit`` records gates exactly as ket's ``Circuit`` does -- same method
names, argument order and validation (``IndexError`` for a qubit out of
range, ``ValueError`` for a repeated operand, as ket's pybind11 module maps
std::out_of_range / std::invalid_argument; src/circuit.cpp:20-40) -- and
lowers them to the flat ``ketgpu_op`` array the C ABI consumes.  Composite
blocks (``append``) are kept as nodes and flattened with ket's wire remap
(src/simulator.cpp:504-511) when the circuit is lowered.
"""
from __future__ import annotations

import enum
from typing import List, Sequence

import numpy as np

from ._lib import OP_DTYPE


class GateType(enum.IntEnum):
    """ket::GateType numbering (include/ket/gate.hpp:16-29)."""
    H = 0
    X = 1
    Y = 2
    Z = 3
    S = 4
    Sdg = 5
    T = 6
    Tdg = 7
    Rx = 8
    Ry = 9
    Rz = 10
    U = 11
    CH = 12
    CX = 13
    CY = 14
    CZ = 15
    CRx = 16
    CRy = 17
    CRz = 18
    CU = 19
    CP = 20
    Swap = 21
    CCX = 22
    CSwap = 23
    Measure = 24
    Barrier = 25
    Composite = 26
    Probe = 27


CLIFFORD = {GateType.H, GateType.X, GateType.Y, GateType.Z, GateType.S, GateType.Sdg,
            GateType.CX, GateType.CY, GateType.CZ, GateType.Swap,
            GateType.Measure, GateType.Barrier, GateType.Probe}


class Gate:
    __slots__ = ("type", "qubits", "params", "label", "definition", "clbit")

    def __init__(self, type_, qubits, params=(), label="", definition=None, clbit=0):
        self.type = GateType(type_)
        self.qubits = list(qubits)
        self.params = list(params)
        self.label = label
        self.definition = definition
        self.clbit = clbit

    def __repr__(self):
        return f"Gate({self.type.name}, {self.qubits}, {self.params})"


class Circuit:
    def __init__(self, n_qubits: int, name: str = ""):
        if n_qubits < 0:
            raise ValueError("n_qubits must be non-negative")
        self._n = int(n_qubits)
        self._nclbits = 0
        self._name = name
        self._gates: List[Gate] = []

    # -- properties (module.cpp:64-66)
    @property
    def n_qubits(self) -> int:
        return self._n

    @property
    def n_clbits(self) -> int:
        return self._nclbits

    @property
    def name(self) -> str:
        return self._name

    @property
    def gates(self) -> List[Gate]:
        return list(self._gates)

    def __repr__(self):
        return f"<ket_b200.Circuit n_qubits={self._n}>"

    # -- validation (circuit.cpp:20-40)
    def _check(self, qubits: Sequence[int]) -> None:
        for q in qubits:
            if not (0 <= q < self._n):
                raise IndexError(f"ket: qubit index {q} is out of range for a {self._n}-qubit circuit")
        for i in range(len(qubits)):
            for j in range(i + 1, len(qubits)):
                if qubits[i] == qubits[j]:
                    raise ValueError(f"ket: a gate cannot act on qubit {qubits[i]} more than once")

    def _add(self, t, qubits, params=()):
        qubits = [int(q) for q in qubits]
        self._check(qubits)
        self._gates.append(Gate(t, qubits, [float(p) for p in params]))

    # -- gates, in GateType order (circuit.hpp:28-66)
    def h(self, qubit): self._add(GateType.H, [qubit])
    def x(self, qubit): self._add(GateType.X, [qubit])
    def y(self, qubit): self._add(GateType.Y, [qubit])
    def z(self, qubit): self._add(GateType.Z, [qubit])
    def s(self, qubit): self._add(GateType.S, [qubit])
    def sdg(self, qubit): self._add(GateType.Sdg, [qubit])
    def t(self, qubit): self._add(GateType.T, [qubit])
    def tdg(self, qubit): self._add(GateType.Tdg, [qubit])
    def rx(self, qubit, theta): self._add(GateType.Rx, [qubit], [theta])
    def ry(self, qubit, theta): self._add(GateType.Ry, [qubit], [theta])
    def rz(self, qubit, theta): self._add(GateType.Rz, [qubit], [theta])
    def u(self, qubit, theta, phi, lam): self._add(GateType.U, [qubit], [theta, phi, lam])
    def ch(self, control, target): self._add(GateType.CH, [control, target])
    def cx(self, control, target): self._add(GateType.CX, [control, target])
    def cy(self, control, target): self._add(GateType.CY, [control, target])
    def cz(self, a, b): self._add(GateType.CZ, [a, b])
    def crx(self, control, target, theta): self._add(GateType.CRx, [control, target], [theta])
    def cry(self, control, target, theta): self._add(GateType.CRy, [control, target], [theta])
    def crz(self, control, target, theta): self._add(GateType.CRz, [control, target], [theta])

    def cu(self, control, target, theta, phi, lam):
        self._add(GateType.CU, [control, target], [theta, phi, lam])

    def cp(self, a, b, lam): self._add(GateType.CP, [a, b], [lam])
    def swap(self, a, b): self._add(GateType.Swap, [a, b])
    def ccx(self, control1, control2, target): self._add(GateType.CCX, [control1, control2, target])
    def cswap(self, control, a, b): self._add(GateType.CSwap, [control, a, b])

    # -- structural ops (circuit.cpp:127-175)
    def barrier(self, qubits=None, label: str = ""):
        if isinstance(qubits, str):
            label, qubits = qubits, None
        qs = list(range(self._n)) if qubits is None else [int(q) for q in qubits]
        self._check(qs)
        self._gates.append(Gate(GateType.Barrier, qs, label=label))

    def measure(self, qubit, clbit):
        self._check([qubit])
        self._nclbits = max(self._nclbits, int(clbit) + 1)
        self._gates.append(Gate(GateType.Measure, [int(qubit)], clbit=int(clbit)))

    def measure_all(self):
        for q in range(self._n):
            self.measure(q, q)

    def probe(self, label: str = ""):
        name = label
        if not name:
            k = sum(1 for g in self._gates if g.type == GateType.Probe)
            name = "ψ" + str(k)
        self._gates.append(Gate(GateType.Probe, list(range(self._n)), label=name))

    def append(self, sub: "Circuit", qubits, name: str = ""):
        qubits = [int(q) for q in qubits]
        if len(qubits) != sub.n_qubits:
            raise ValueError(f"ket: append expects {sub.n_qubits} qubits, got {len(qubits)}")
        self._check(qubits)
        block = name or sub.name or "circ"
        self._gates.append(Gate(GateType.Composite, qubits, label=block, definition=sub))

    def decompose(self) -> "Circuit":
        out = Circuit(self._n, self._name)
        out._nclbits = self._nclbits
        for g in self._gates:
            if g.type == GateType.Composite and g.definition is not None:
                for sg in g.definition._gates:
                    ng = Gate(sg.type, [g.qubits[q] for q in sg.qubits], sg.params, sg.label,
                              sg.definition, sg.clbit)
                    out._gates.append(ng)
            else:
                out._gates.append(g)
        return out

    # -- lowering ------------------------------------------------------------
    def flat_gates(self, wire=None):
        """Gates with composites expanded recursively (simulator.cpp:504-511)."""
        wire = list(range(self._n)) if wire is None else wire
        out = []
        for g in self._gates:
            if g.type == GateType.Composite:
                sub_wire = [wire[q] for q in g.qubits]
                out.extend(g.definition.flat_gates(sub_wire))
            else:
                out.append(Gate(g.type, [wire[q] for q in g.qubits], g.params, g.label, None, g.clbit))
        return out

    def to_ops(self) -> np.ndarray:
        gates = self.flat_gates()
        ops = np.zeros(len(gates), dtype=OP_DTYPE)
        for i, g in enumerate(gates):
            ops[i]["type"] = int(g.type)
            if g.type in (GateType.Barrier, GateType.Probe):
                ops[i]["nq"] = 0
            elif g.type == GateType.Measure:
                ops[i]["nq"] = 1
                ops[i]["q"][0] = g.qubits[0]
                ops[i]["q"][1] = g.clbit
            else:
                ops[i]["nq"] = len(g.qubits)
                for j, q in enumerate(g.qubits):
                    ops[i]["q"][j] = q
                for j, p in enumerate(g.params):
                    ops[i]["p"][j] = p
        return ops

    def is_clifford(self) -> bool:
        """backend.cpp:16-47: only H X Y Z S Sdg CX CY CZ Swap (+ structural)."""
        for g in self._gates:
            if g.type == GateType.Composite:
                if g.definition is None or not g.definition.is_clifford():
                    return False
            elif g.type not in CLIFFORD:
                return False
        return True

    def measurements(self):
        """(qubit, clbit) of every Measure, in circuit order (backend.cpp:72-80)."""
        return [(g.qubits[0], g.clbit) for g in self.flat_gates() if g.type == GateType.Measure]
