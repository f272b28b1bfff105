"""ket's own C++ API, unchanged, running on the B200 backend.

oracle/_ref/libket_dropin.so is ket's off-path translation units (circuit,
DAG, state, QASM, backend dispatch, stabilizer) linked with
ket_b200/host/ket_statevector_gpu.cpp in place of ket's state-vector units;
oracle/_ref/libket_ref.so is ket itself.  The same shim drives both through
ket::run / expval / measure / sample / simulate, so every difference below
is the backend's.
"""
import math
import os

import numpy as np
import pytest

from oracle.oracle import ARITY, DROPIN_SO, GATES, NPARAMS, REF_SO, make_ops

pytestmark = pytest.mark.skipif(not (os.path.exists(REF_SO) and os.path.exists(DROPIN_SO)),
                                reason="ket sources were not available to build the drop-in")


def _libs():
    from oracle.oracle import Reference
    return Reference(dropin=False), Reference(dropin=True)


def _random_ops(n, count, seed, gates=GATES[:24]):
    rng = np.random.default_rng(seed)
    gs = []
    for _ in range(count):
        g = gates[int(rng.integers(len(gates)))]
        qs = rng.choice(n, ARITY[g], replace=False).tolist()
        ps = rng.uniform(0, 2 * math.pi, NPARAMS.get(g, 0)).tolist()
        gs.append((g, qs, ps))
    return make_ops(gs)


def test_dropin_library_loads_and_exports_the_shim():
    import ctypes
    lib = ctypes.CDLL(DROPIN_SO)
    for name in ("ref_run", "ref_expval_sum", "ref_sample", "ref_simulate_sample", "ref_is_clifford"):
        assert hasattr(lib, name)


def test_routing_decisions_are_kets_own():
    R, D = _libs()
    cliff = make_ops([("H", [0]), ("CX", [0, 1]), ("S", [1]), ("Swap", [1, 2]), ("Measure", [0, 0])])
    non = make_ops([("H", [0]), ("T", [0]), ("Measure", [0, 0])])
    for ops in (cliff, non):
        assert R.is_clifford(3, ops) == D.is_clifford(3, ops)
        assert R.chosen_method(3, ops) == D.chosen_method(3, ops)


@pytest.mark.gpu
def test_run_matches_ket():
    R, D = _libs()
    for n, count, seed in [(3, 40, 1), (8, 200, 2), (12, 300, 3)]:
        ops = _random_ops(n, count, seed)
        assert np.abs(R.run(n, ops) - D.run(n, ops)).max() < 1e-12


@pytest.mark.gpu
def test_run_with_probes_matches_ket():
    R, D = _libs()
    ops = make_ops([("H", [0]), ("Probe", []), ("CX", [0, 1]), ("T", [1]), ("Probe", []), ("Rx", [2], [0.4])])
    fr, pr = R.run_with_probes(3, ops)
    fd, pd = D.run_with_probes(3, ops)
    assert len(pr) == len(pd) == 2
    assert np.abs(fr - fd).max() < 1e-12 and np.abs(pr - pd).max() < 1e-12


@pytest.mark.gpu
def test_expval_matches_ket():
    R, D = _libs()
    n = 9
    ops = _random_ops(n, 150, 4)
    st = R.run(n, ops)
    g = np.random.default_rng(5)
    terms = [(float(g.standard_normal()), "".join("IXYZ"[i] for i in g.integers(0, 4, n))) for _ in range(12)]
    assert abs(R.expval_sum(n, st, terms) - D.expval_sum(n, st, terms)) < 1e-12
    for _, p in terms[:4]:
        assert abs(R.expval(n, st, p) - D.expval(n, st, p)) < 1e-12
    for method in (0, 1):
        assert abs(R.expval_circuit(n, ops, terms, method) - D.expval_circuit(n, ops, terms, method)) < 1e-12
    with pytest.raises(ValueError):
        D.expval(n, st, "ZZ")


@pytest.mark.gpu
def test_measure_and_sample_match_ket():
    R, D = _libs()
    n = 5
    ops = _random_ops(n, 60, 6)
    st = R.run(n, ops)
    # n = 5 is a single 32-amplitude segment: the tree sampler is ket's scan
    assert np.array_equal(R.measure(n, st, 42, 300), D.measure(n, st, 42, 300))
    circ = np.concatenate([ops, make_ops([("Measure", [0, 0]), ("Measure", [3, 1]), ("Measure", [4, 2])])])
    for method in (0, 1):
        assert np.array_equal(R.sample(n, circ, 7, 50, method), D.sample(n, circ, 7, 50, method))
    # one Simulation, many shots: the GPU backend answers from HBM
    a, name_r = R.sample(n, circ, 9, 500, method=1, evolve_once=True)
    b, name_d = D.sample(n, circ, 9, 500, method=1, evolve_once=True)
    assert np.array_equal(a, b) and name_r == name_d == "state vector"


@pytest.mark.gpu
def test_clifford_circuits_stay_on_kets_stabilizer():
    R, D = _libs()
    ops = make_ops([("H", [0]), ("CX", [0, 1]), ("CX", [1, 2]), ("S", [2]), ("Measure", [0, 0]),
                    ("Measure", [1, 1]), ("Measure", [2, 2])])
    a, name_r = R.sample(3, ops, 11, 200, method=0, evolve_once=True)
    b, name_d = D.sample(3, ops, 11, 200, method=0, evolve_once=True)
    assert name_r == name_d == "stabilizer"
    assert np.array_equal(a, b)


def _qasm_programs():
    import json
    with open(os.path.join(os.path.dirname(__file__), "golden", "qasm.json")) as f:
        return json.load(f)["programs"]


def test_qasm_reads_and_writes_through_kets_own_parser():
    """ket::from_qasm / to_qasm are ket's, unchanged, in the drop-in build."""
    _, D = _libs()
    for prog in _qasm_programs():
        assert D.qasm_roundtrip(prog["source"]) == prog["to_qasm"], prog["name"]


@pytest.mark.gpu
def test_qasm_programs_run_on_the_gpu_through_ket():
    """ket's parser feeding ket::run on the B200 backend."""
    _, D = _libs()
    for prog in _qasm_programs():
        if "state" not in prog:
            continue
        r = D.qasm_parse(prog["source"])
        want = np.array([complex(float.fromhex(a), float.fromhex(b)) for a, b in prog["state"]])
        assert np.abs(D.run(r["n_qubits"], r["ops"]) - want).max() < 1e-12, prog["name"]


@pytest.mark.gpu
def test_stepper_steps_and_seeks_like_kets():
    """ket::Stepper on the B200 backend against ket's own (tests/test_stepper.cpp:51-96
    in ket): the state at every position when stepping to the end, then seeks
    forward, backward, to the same place and past the end."""
    R, D = _libs()
    rng = np.random.default_rng(17)
    gs = []
    for i in range(40):
        g = GATES[int(rng.integers(24))]
        qs = rng.choice(5, ARITY[g], replace=False).tolist()
        gs.append((g, qs, rng.uniform(0, 2 * math.pi, NPARAMS.get(g, 0)).tolist()))
        if i % 9 == 4:
            gs.append(("Barrier", []))
        if i % 13 == 6:
            gs.append(("Measure", [int(rng.integers(5)), i % 3]))
    ops = make_ops(gs)
    want, got = R.stepper_walk(5, ops), D.stepper_walk(5, ops)
    assert want.shape == got.shape == (len(ops) + 1, 32)
    assert np.abs(want - got).max() < 1e-12
    size = len(ops)
    seq = [size, 3, 0, size - 1, 5, 5, size + 10, 1, size // 2]
    (sw, pw), (sg, pg) = R.stepper_seek(5, ops, seq), D.stepper_seek(5, ops, seq)
    assert pw.tolist() == pg.tolist() == [min(k, size) for k in seq]
    assert np.abs(sw - sg).max() < 1e-12


@pytest.mark.gpu
def test_stabilizer_equals_gpu_statevector_on_cliffords():
    """ket's tableau and the B200 state vector agree on random Clifford
    circuits for every Pauli string (ket's own check,
    tests/test_stabilizer.cpp:91-106, seed 1234, 1e-9), both reached through
    ket's expval(Circuit, PauliSum, Method)."""
    import itertools
    _, D = _libs()
    clifford = ["H", "S", "Sdg", "X", "Y", "Z", "CX", "CY", "CZ", "Swap"]
    n = 3
    paulis = ["".join(p) for p in itertools.product("IXYZ", repeat=n)]
    for seed in (1234, 1235, 1236, 1237):
        ops = _random_ops(n, 40, seed, gates=clifford)
        for p in paulis:
            stab = D.expval_circuit(n, ops, [(1.0, p)], method=2)
            sv = D.expval_circuit(n, ops, [(1.0, p)], method=1)
            assert abs(stab - sv) < 1e-9, (seed, p)


@pytest.mark.gpu
def test_simulation_sample_draws_from_one_tree(oracle):
    """ket's StateVectorSimulation::sample (statevector.cpp:33-42), called once
    per shot as ket's CLI does (cli/commands.cpp:159-166): 10^4 draws on a
    5-qubit register are ket's own draws bit for bit (one 32-amplitude
    segment: the tree is ket's scan), and on 12 qubits every draw comes from
    one sampling tree built once for the state, equal to the oracle's tree
    sampler fed the same std::mt19937 stream."""
    from ket_b200 import _lib
    R, D = _libs()
    n = 5
    ops = np.concatenate([_random_ops(n, 60, 31), make_ops([("Measure", [q, q]) for q in range(n)])])
    a, _ = R.sample(n, ops, 77, 10000, method=1, evolve_once=True)
    b, _ = D.sample(n, ops, 77, 10000, method=1, evolve_once=True)
    assert np.array_equal(a, b)

    n = 12
    body = _random_ops(n, 150, 32)
    ops = np.concatenate([body, make_ops([("Measure", [q, q]) for q in range(n)])])
    builds = _lib.lib.ketgpu_sample_tree_builds()
    got, _ = D.sample(n, ops, 78, 10000, method=1, evolve_once=True)
    assert _lib.lib.ketgpu_sample_tree_builds() - builds == 1
    st = D.run(n, body)
    idx = oracle.sample_tree(n, st, oracle.uniforms(78, 10000))
    want = ((idx[:, None] >> np.arange(n, dtype=np.uint64)) & np.uint64(1)).astype(np.int32)
    assert np.array_equal(got, want)
