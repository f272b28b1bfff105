"""Generate the golden fixtures under tests/golden from ket itself.

Run in a checkout where the reference sources are available:
    make -C oracle ref          # builds oracle/_ref/libket_ref.so from ket's sources
    python tests/golden/make_golden.py
Every fixture is the output of ket's own code (ket::run, ket::expval,
ket::measure, ket::sample, ket::from_qasm, ket::to_qasm, ket::State::print)
called through oracle/ref_shim.cpp; the circuits are seeded and stored next
to the outputs.
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import ARITY, CODE, GATES, NPARAMS, Reference, make_ops  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def gate_battery():
    """Each unitary gate on a 4-qubit register prepared in a generic state."""
    prep = [("H", [0]), ("H", [1]), ("H", [2]), ("H", [3]), ("T", [0]), ("Rx", [1], [0.3]),
            ("Ry", [2], [1.1]), ("Rz", [3], [2.2]), ("CX", [0, 2]), ("CZ", [1, 3])]
    cases = []
    for g in GATES[:24]:
        a = ARITY[g]
        for qs in ([0, 1, 2][:a], [3, 1, 0][:a], [2, 3, 1][:a]):
            params = [0.7, 1.9, 2.6][:NPARAMS.get(g, 0)]
            cases.append((g, qs, params, prep + [(g, qs, params)]))
    return cases


def random_ops(n, count, seed):
    rng = np.random.default_rng(seed)
    gs = []
    for _ in range(count):
        g = GATES[int(rng.integers(24))]
        qs = rng.choice(n, ARITY[g], replace=False).tolist()
        ps = rng.uniform(0, 2 * math.pi, NPARAMS.get(g, 0)).tolist()
        gs.append((g, qs, ps))
    return make_ops(gs)


def brickwork_ops(n, depth, seed):
    sys.path.insert(0, ROOT)
    from ket_b200.workloads import MT19937
    rng = MT19937(seed)
    gs = []
    for layer in range(depth):
        for q in range(n):
            th, ph, la = (rng.uniform(0.0, 2 * math.pi) for _ in range(3))
            gs.append(("U", [q], [th, ph, la]))
        for a in range(layer % 2, n - 1, 2):
            gs.append(("CX", [a, a + 1]))
    return make_ops(gs)


def _hexops(ops):
    return [[int(o["type"]), int(o["nq"])] + [int(v) for v in o["q"]] + [float(v).hex() for v in o["p"]]
            for o in ops]


def qasm_golden(R):
    """ket::from_qasm / ket::to_qasm on the programs of qasm_programs.py:
    the parsed circuit (flattened), its to_qasm text, ket::run's state for
    the programs without measurements, the rejections, and to_qasm's angle
    formatting."""
    sys.path.insert(0, OUT)
    from qasm_programs import ANGLES, ERRORS, PROGRAMS
    progs = []
    for name, src in PROGRAMS:
        r = R.qasm_parse(src)
        entry = {"name": name, "source": src, "n_qubits": r["n_qubits"], "n_clbits": r["n_clbits"],
                 "n_top": r["n_top"], "ops": _hexops(r["ops"]), "to_qasm": R.qasm_roundtrip(src)}
        ops = r["ops"]
        finite = bool(np.isfinite(ops["p"]).all()) if len(ops) else True
        if finite and not (ops["type"] == CODE["Measure"]).any() and r["n_qubits"] <= 8:
            st = R.run(r["n_qubits"], ops)
            entry["state"] = [[float(z.real).hex(), float(z.imag).hex()] for z in st]
        progs.append(entry)
    errs = []
    for name, src in ERRORS:
        try:
            R.qasm_parse(src)
        except Exception as e:  # noqa: BLE001 -- the rejection is the fixture
            errs.append({"name": name, "source": src, "kind": type(e).__name__, "message": str(e)})
        else:
            raise AssertionError(f"ket accepted {name}")
    angles = []
    for a in ANGLES:
        ops = make_ops([("Rz", [0], [a]), ("U", [0], [a, -a, 2 * a]), ("CP", [0, 1], [a])])
        angles.append({"angle": float(a).hex(), "to_qasm": R.to_qasm(2, ops)})
    mixed = make_ops([("H", [0]), ("CU", [1, 2], [0.5, math.pi / 3, -math.pi]), ("Measure", [2, 3]),
                      ("Barrier", []), ("Probe", []), ("CSwap", [0, 1, 2]), ("Measure", [0, 0])])
    with open(os.path.join(OUT, "qasm.json"), "w") as f:
        json.dump({"programs": progs, "errors": errs, "angles": angles,
                   "mixed": {"n": 3, "ops": _hexops(mixed), "to_qasm": R.to_qasm(3, mixed)}}, f, indent=1)


def state_print_golden(R):
    """ket::State::print on generic and edge-valued states."""
    special = np.array([0.0, -0.0, 1.0, -1.0, 1j, -1j, 0.5 - 0.25j, 1e-30 + 1e30j,
                        -0.0 + 0.3j, 0.1 - 0.0j, 123456789.0, 1.5e-7 - 2.25e-8j, 0.25 + 1e-300j,
                        -7.125 + 7.125j, 2.0 ** -20, 3.0 - 1e20j])
    rng = np.random.default_rng(11)
    cases = [(0, np.array([1.0 + 0.0j])), (1, np.array([0.6, -0.8j])), (4, special),
             (6, rng.standard_normal(64) + 1j * rng.standard_normal(64))]
    out = [{"n": n, "state": [[float(z.real).hex(), float(z.imag).hex()] for z in st],
            "text": R.state_print(n, st)} for n, st in cases]
    with open(os.path.join(OUT, "state_print.json"), "w") as f:
        json.dump(out, f, indent=1, ensure_ascii=False)


def main():
    R = Reference()
    # 1. gate battery: every gate, three operand orders, 4 qubits
    names, states, opsl = [], [], []
    for g, qs, ps, circ in gate_battery():
        ops = make_ops(circ)
        names.append(f"{g}:{','.join(map(str, qs))}")
        states.append(R.run(4, ops))
        opsl.append(ops)
    np.savez_compressed(os.path.join(OUT, "gate_battery.npz"), names=np.array(names),
                        states=np.stack(states), ops=np.stack(opsl))

    # 2. random mixed circuits through ket::run (its Fuser engaged)
    rnd = {}
    for n, count, seed in [(6, 120, 1), (10, 300, 2), (12, 400, 3)]:
        ops = random_ops(n, count, seed)
        rnd[f"ops_{n}"] = ops
        rnd[f"state_{n}"] = R.run(n, ops)
    np.savez_compressed(os.path.join(OUT, "random_mixed.npz"), **rnd)

    # 3. the 20-qubit depth-20 U + CX brick wall (seed 1234): summary of ket::run
    ops = brickwork_ops(20, 20, 1234)
    st = R.run(20, ops)
    rng = np.random.default_rng(5)
    idx = np.sort(rng.choice(1 << 20, 4096, replace=False))
    np.savez_compressed(os.path.join(OUT, "brickwork_20q_d20.npz"), ops=ops, head=st[:4096],
                        idx=idx, sampled=st[idx], norm=np.array([np.vdot(st, st).real]),
                        abs_sum=np.array([np.abs(st).sum()]))

    # 4. Pauli expectations (single strings and a sum) on the 10-qubit state
    s10 = rnd["state_10"]
    g = np.random.default_rng(9)
    paulis = ["".join("IXYZixyz"[i] for i in g.integers(0, 8, 10)) for _ in range(40)]
    vals = np.array([R.expval(10, s10, p) for p in paulis])
    coeffs = g.standard_normal(40)
    total = R.expval_sum(10, s10, list(zip(coeffs.tolist(), paulis)))
    np.savez_compressed(os.path.join(OUT, "expval.npz"), paulis=np.array(paulis), values=vals,
                        coeffs=coeffs, total=np.array([total]))

    # 5. measure: ket::measure draws on one mt19937 stream, and the stream itself
    m = {}
    for seed in (42, 7, 2024):
        m[f"outcomes_{seed}"] = R.measure(10, s10, seed, 2000)
        m[f"uniforms_{seed}"] = R.uniforms(seed, 2000)
    np.savez_compressed(os.path.join(OUT, "measure.npz"), **m)

    # 6. sample: ket::sample with explicit StateVector and Auto methods
    circ = make_ops([("H", [0]), ("CX", [0, 1]), ("T", [1]), ("H", [2]), ("CCX", [0, 2, 3]),
                     ("Measure", [0, 0]), ("Measure", [1, 2]), ("Measure", [3, 1])])
    sv = R.sample(4, circ, 123, 200, method=1)
    au = R.sample(4, circ, 123, 200, method=0)
    np.savez_compressed(os.path.join(OUT, "sample.npz"), ops=circ, statevector=sv, auto=au)
    # 7. OpenQASM: ket::from_qasm and ket::to_qasm
    qasm_golden(R)
    # 8. State::print
    state_print_golden(R)
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    if sys.argv[1:] == ["qasm"]:  # only the OpenQASM and State::print fixtures
        qasm_golden(Reference())
        state_print_golden(Reference())
    else:
        main()
