"""ket's API-level contract, run on the GPU through ket_b200 (the Python
mirror of ket's module).  Cases follow ket's tests/test_simulator.cpp,
test_observable.cpp, test_measurement.cpp and tests/python/test_ket.py."""
import math

import numpy as np
import pytest

import ket_b200 as ket

pytestmark = pytest.mark.gpu

R = 1.0 / math.sqrt(2.0)
TOL = 1e-12


def amp(s, i, want):
    assert abs(s[i] - want) < TOL, (i, s[i], want)


@pytest.fixture(autouse=True, params=["greedy", "none", "reference"])
def mode(request):
    ket.set_options(precision="c128", fusion=request.param)
    yield request.param
    ket.set_options(precision="c128", fusion="greedy")


def test_empty_circuit_is_ground_state():
    s = ket.run(ket.Circuit(2))
    assert len(s) == 4
    amp(s, 0, 1)
    for i in (1, 2, 3):
        amp(s, i, 0)


def test_bell_and_cnot():
    c = ket.Circuit(2)
    c.h(0)
    c.cx(0, 1)
    s = ket.run(c)
    amp(s, 0, R)
    amp(s, 3, R)
    amp(s, 1, 0)
    c = ket.Circuit(2)
    c.x(0)
    c.cx(0, 1)
    amp(ket.run(c), 3, 1)


def test_phases_and_rotations():
    c = ket.Circuit(1)
    c.x(0)
    c.s(0)
    amp(ket.run(c), 1, 1j)
    c = ket.Circuit(1)
    c.x(0)
    c.t(0)
    amp(ket.run(c), 1, complex(R, R))
    c = ket.Circuit(1)
    c.x(0)
    c.z(0)
    amp(ket.run(c), 1, -1)
    c = ket.Circuit(1)
    c.y(0)
    amp(ket.run(c), 1, 1j)
    c = ket.Circuit(1)
    c.rx(0, math.pi)
    amp(ket.run(c), 1, -1j)
    c = ket.Circuit(1)
    c.ry(0, math.pi / 2)
    s = ket.run(c)
    amp(s, 0, R)
    amp(s, 1, R)
    c = ket.Circuit(1)
    c.rz(0, math.pi / 2)
    amp(ket.run(c), 0, complex(math.cos(math.pi / 4), -math.sin(math.pi / 4)))


def test_controlled_and_three_qubit_gates():
    c = ket.Circuit(3)
    c.x(0)
    c.x(1)
    c.ccx(0, 1, 2)
    amp(ket.run(c), 7, 1)
    c = ket.Circuit(3)
    c.x(0)
    c.x(1)
    c.cswap(0, 1, 2)
    amp(ket.run(c), 0b101, 1)
    c = ket.Circuit(2)
    c.x(0)
    c.swap(0, 1)
    amp(ket.run(c), 2, 1)
    c = ket.Circuit(2)
    c.x(0)
    c.x(1)
    c.cz(0, 1)
    amp(ket.run(c), 3, -1)
    c = ket.Circuit(2)
    c.x(0)
    c.x(1)
    c.cp(0, 1, math.pi / 2)
    amp(ket.run(c), 3, 1j)
    c = ket.Circuit(2)
    c.x(0)
    c.ch(0, 1)
    s = ket.run(c)
    amp(s, 1, R)
    amp(s, 3, R)
    c = ket.Circuit(2)
    c.x(0)
    c.cy(0, 1)
    amp(ket.run(c), 3, 1j)
    c = ket.Circuit(2)
    c.x(0)
    c.crx(0, 1, math.pi)
    amp(ket.run(c), 3, -1j)


def test_swap_equals_three_cnots():
    a = ket.Circuit(3)
    b = ket.Circuit(3)
    for c in (a, b):
        c.h(0)
        c.t(0)
        c.ry(1, 0.4)
    a.swap(0, 1)
    b.cx(0, 1)
    b.cx(1, 0)
    b.cx(0, 1)
    assert np.abs(ket.run(a).to_numpy() - ket.run(b).to_numpy()).max() < TOL


def test_u_special_cases():
    c = ket.Circuit(1)
    c.u(0, math.pi / 2, 0, math.pi)  # = H
    s = ket.run(c)
    amp(s, 0, R)
    amp(s, 1, R)


def test_barrier_and_probes():
    c = ket.Circuit(2)
    c.h(0)
    c.probe("a")
    c.barrier()
    c.cx(0, 1)
    c.probe()
    r = ket.run_with_probes(c)
    assert [p[0] for p in r.probes] == ["a", "ψ1"]
    amp(r.probes[0][1], 1, R)
    amp(r.final, 3, R)


def test_composite_blocks_flatten_like_decompose():
    sub = ket.Circuit(2, "bell")
    sub.h(0)
    sub.cx(0, 1)
    c = ket.Circuit(3)
    c.append(sub, [2, 0])
    c.t(2)
    a = ket.run(c).to_numpy()
    b = ket.run(c.decompose()).to_numpy()
    assert np.abs(a - b).max() < TOL
    amp(ket.run(c), 0b101, complex(R * R, R * R))


def test_errors_match_ket():
    c = ket.Circuit(2)
    with pytest.raises(IndexError):
        c.h(2)
    with pytest.raises(ValueError):
        c.cx(1, 1)
    with pytest.raises(ValueError):
        ket.expval(ket.run(c), "Z")
    with pytest.raises(IndexError):
        _ = ket.run(ket.Circuit(1))[99]
    with pytest.raises(ValueError):
        ket.sample(c, method="nope")


def test_observables():
    c = ket.Circuit(2)
    c.h(0)
    c.cx(0, 1)
    s = ket.run(c)
    assert abs(ket.expval(s, "ZZ") - 1) < TOL
    assert abs(ket.expval(s, "XX") - 1) < TOL
    assert abs(ket.expval(s, "YY") + 1) < TOL
    assert abs(ket.expval(s, "ZI")) < TOL
    c = ket.Circuit(2)
    c.x(1)
    s = ket.run(c)
    assert abs(ket.expval(s, "ZI") + 1) < TOL
    assert abs(ket.expval(s, "IZ") - 1) < TOL
    h = [(0.5, "ZI"), (0.25, "IZ")]
    assert abs(ket.expval(s, h) - (-0.5 + 0.25)) < TOL
    # circuit overload on a non-Clifford circuit runs the state vector
    c = ket.Circuit(1)
    c.h(0)
    c.t(0)
    assert abs(ket.expval(c, "X") - R) < TOL


def test_measurement():
    c = ket.Circuit(2)
    c.h(0)
    c.cx(0, 1)
    s = ket.run(c)
    a = [ket.measure(s, seed=42) for _ in range(5)]
    assert a == [ket.measure(s, seed=42) for _ in range(5)]
    assert {ket.measure(s, seed=k) for k in range(200)} == {0, 3}
    for _ in range(20):
        assert ket.measure(ket.run(ket.Circuit(1))) == 0


def test_many_shot_sampling_statistics():
    c = ket.Circuit(2)
    c.h(0)
    c.cx(0, 1)
    c.t(1)
    c.measure_all()
    creg = ket.sample_shots(c, 10000, seed=42)
    counts = {}
    for row in creg.tolist():
        counts[tuple(row)] = counts.get(tuple(row), 0) + 1
    assert set(counts) == {(0, 0), (1, 1)}
    assert 4800 < counts[(0, 0)] < 5200


def test_sample_statevector_matches_ket(golden):
    g = golden("sample")
    c = ket.Circuit(4)
    c.h(0)
    c.cx(0, 1)
    c.t(1)
    c.h(2)
    c.ccx(0, 2, 3)
    c.measure(0, 0)
    c.measure(1, 2)
    c.measure(3, 1)
    want = g["statevector"]
    # ket::sample(circuit, rng) draws one uniform per call from the same
    # stream; sample_shots consumes the stream in the same order.
    got = ket.sample_shots(c, len(want), seed=123)
    assert np.array_equal(got, want)
    assert ket.chosen_method(c) == "statevector" and not ket.is_clifford(c)


def test_clifford_routing_decisions():
    c = ket.Circuit(3)
    c.h(0)
    c.cx(0, 1)
    c.s(2)
    c.measure_all()
    assert ket.is_clifford(c)
    assert ket.chosen_method(c) == "stabilizer"
    c.t(1)
    assert not ket.is_clifford(c)
    with pytest.raises(ValueError):
        ket.sample(c, seed=1, method="stabilizer")


def test_edge_cases_like_ket():
    """Empty Hamiltonian, negative coefficients (test_observable.cpp:60-74),
    the 0- and 1-qubit registers, and zero shots."""
    c = ket.Circuit(2)
    c.h(0)
    c.cx(0, 1)
    s = ket.run(c)
    assert abs(ket.expval(s, [(0.5, "ZZ"), (0.5, "XX")]) - 1.0) < TOL
    assert abs(ket.expval(s, [(2.0, "ZZ"), (-1.0, "YY")]) - 3.0) < TOL
    assert ket.expval(s, []) == 0.0
    # a register of no qubits holds one amplitude, 1
    s0 = ket.run(ket.Circuit(0))
    assert len(s0) == 1
    amp(s0, 0, 1)
    # one qubit, every single-qubit gate in a row, against the oracle's matrices
    c1 = ket.Circuit(1)
    c1.h(0)
    c1.t(0)
    c1.ry(0, 0.3)
    c1.s(0)
    c1.rz(0, 1.1)
    c1.u(0, 0.2, 0.4, 0.6)
    s1 = ket.run(c1)
    assert abs(abs(s1[0]) ** 2 + abs(s1[1]) ** 2 - 1) < TOL
    # zero shots give an empty sample
    c2 = ket.Circuit(2)
    c2.h(0)
    c2.t(1)
    c2.measure_all()
    assert len(ket.sample_shots(c2, 0, seed=1)) == 0


def test_run_reuses_its_device_state(golden):
    """ketgpu_run keeps its device state between calls: every call still
    starts from |0...0>, whatever size, precision or release came before."""
    import ctypes as ct
    from ket_b200 import _lib
    g = golden("random_mixed")

    def run(n, precision):
        out = np.zeros(1 << n, dtype=np.complex128)
        opt = ket.make_options(precision, "greedy", 5, True)
        ops = g[f"ops_{n}"]
        _lib.check(_lib.lib.ketgpu_run(n, ops.ctypes.data, len(ops), ct.byref(opt), out.ctypes.data))
        return out

    tol = {"c128": 1e-12, "c64": 1e-5}
    for n, precision in [(12, "c128"), (12, "c128"), (10, "c128"), (12, "c64"), (12, "c64"), (12, "c128")]:
        assert np.abs(run(n, precision) - g[f"state_{n}"]).max() < tol[precision], (n, precision)
    _lib.check(_lib.lib.ketgpu_release_cache())
    _lib.check(_lib.lib.ketgpu_release_cache())
    assert np.abs(run(12, "c64") - g["state_12"]).max() < 1e-5


def test_repeated_runs_are_bit_identical(golden):
    """The same circuit gives the same bits every time and whatever the thread
    setting, as ket demands of its parallel runs (EXPECT_DOUBLE_EQ,
    tests/test_parallelism.cpp:70-85): no reduction on the path depends on
    scheduling."""
    import ctypes as ct
    from ket_b200 import _lib
    ops = golden("random_mixed")["ops_12"]
    try:
        for precision in ("c128", "c64"):
            opt = ket.make_options(precision, "greedy", 5, True)
            runs = []
            for threads in (1, 8, 0, 1):
                ket.set_num_threads(threads)
                out = np.zeros(1 << 12, dtype=np.complex128)
                _lib.check(_lib.lib.ketgpu_run(12, ops.ctypes.data, len(ops), ct.byref(opt), out.ctypes.data))
                runs.append(out)
            assert all(np.array_equal(r, runs[0]) for r in runs[1:]), precision
    finally:
        ket.set_num_threads(1)
