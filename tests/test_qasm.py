"""OpenQASM ingest: ket_b200.from_qasm / to_qasm against ket's own parser and
writer (bindings/qasm/qasm.cpp).

tests/golden/qasm.json holds what ket::from_qasm and ket::to_qasm did with
the programs of tests/golden/qasm_programs.py: the parsed circuit (gates
flattened through composite wire maps; parameters as hex floats, compared
bit-exactly), the to_qasm text (compared byte for byte), and each rejected
program's exception type and message.  The GPU half (ket::run's state of
each program) is in test_gpu_qasm.py.
"""
import json
import math
import os

import pytest

import ket_b200 as ket
from ket_b200.circuit import GateType

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "qasm.json")


@pytest.fixture(scope="module")
def fixture():
    with open(GOLDEN) as f:
        return json.load(f)


def flat_records(c):
    """Our circuit in the fixture's record form: type, width, the first three
    qubits (a measure's classical bit in the second), three parameters."""
    out = []
    for g in c.flat_gates():
        q = list(g.qubits[:3])
        if g.type == GateType.Measure:
            q = [g.qubits[0], g.clbit]
        q += [0] * (3 - len(q))
        p = list(g.params[:3]) + [0.0] * (3 - len(g.params[:3]))
        out.append([int(g.type), len(g.qubits)] + q + [float(v).hex() for v in p])
    return out


def test_programs_parse_like_ket(fixture):
    for prog in fixture["programs"]:
        c = ket.from_qasm(prog["source"])
        assert c.n_qubits == prog["n_qubits"], prog["name"]
        assert c.n_clbits == prog["n_clbits"], prog["name"]
        assert len(c.gates) == prog["n_top"], prog["name"]
        assert flat_records(c) == prog["ops"], prog["name"]


def test_to_qasm_writes_like_ket(fixture):
    for prog in fixture["programs"]:
        assert ket.to_qasm(ket.from_qasm(prog["source"])) == prog["to_qasm"], prog["name"]


def test_rejections_match_ket(fixture):
    kinds = {"RuntimeError": RuntimeError, "ValueError": ValueError, "IndexError": IndexError}
    for err in fixture["errors"]:
        with pytest.raises(kinds[err["kind"]]) as info:
            ket.from_qasm(err["source"])
        assert str(info.value) == err["message"], err["name"]


def test_angle_text_like_ket(fixture):
    for case in fixture["angles"]:
        a = float.fromhex(case["angle"])
        c = ket.Circuit(2)
        c.rz(0, a)
        c.u(0, a, -a, 2 * a)
        c.cp(0, 1, a)
        assert ket.to_qasm(c) == case["to_qasm"], case["angle"]


def test_structural_ops_written_like_ket(fixture):
    c = ket.Circuit(3)
    c.h(0)
    c.cu(1, 2, 0.5, math.pi / 3, -math.pi)
    c.measure(2, 3)
    c.barrier()
    c.probe()
    c.cswap(0, 1, 2)
    c.measure(0, 0)
    assert ket.to_qasm(c) == fixture["mixed"]["to_qasm"]


def test_round_trip_keeps_the_circuit(fixture):
    """from_qasm(to_qasm(c)) rebuilds c: same gates, angles to the 15
    significant digits to_qasm writes."""
    for prog in fixture["programs"]:
        if any(not math.isfinite(float.fromhex(p)) for op in prog["ops"] for p in op[5:]):
            continue
        back = flat_records(ket.from_qasm(prog["to_qasm"]))
        assert len(back) == len(prog["ops"]), prog["name"]
        for got, want in zip(back, prog["ops"]):
            assert got[:5] == want[:5], prog["name"]
            for g, w in zip(got[5:], want[5:]):
                assert abs(float.fromhex(g) - float.fromhex(w)) <= 1e-14 * max(1.0, abs(float.fromhex(w)))


def test_composites_are_named_blocks():
    c = ket.from_qasm('qreg q[3]; gate pair(a) x, y { rx(a) x; cz x, y; } pair(0.5) q[2], q[0];')
    (g,) = c.gates
    assert g.type == GateType.Composite and g.label == "pair" and g.qubits == [2, 0]
    assert g.definition.n_qubits == 2 and g.definition.name == "pair"
    # the same name with another body is written as a second definition
    c2 = ket.from_qasm('qreg q[2]; gate r(a) x { rx(a) x; } r(0.5) q[0]; r(0.25) q[1]; r(0.5) q[1];')
    text = ket.to_qasm(c2)
    assert "gate r q0 {" in text and "gate r_2 q0 {" in text
    assert text.endswith("r q[0];\nr_2 q[1];\nr q[1];\n")


def test_state_print_like_ket():
    """State.print / str(State) write what ket::State::print writes
    (tests/golden/state_print.json)."""
    import numpy as np
    from ket_b200.api import State
    with open(os.path.join(os.path.dirname(__file__), "golden", "state_print.json")) as f:
        cases = json.load(f)
    for case in cases:
        amps = np.array([complex(float.fromhex(a), float.fromhex(b)) for a, b in case["state"]])
        assert State(amps).print() == case["text"], case["n"]
        assert str(State(amps)) == case["text"]
