"""Parity of the CUDA path with the oracle and ket's golden outputs.

Tolerances (written here, used throughout):
  * complex128 mode: 1e-12 max-abs per amplitude (ket's own kTol,
    tests/test_simulator.cpp:9);
  * complex64 mode: 1e-5 max-abs per amplitude and fidelity > 1 - 1e-6.
"""
import ctypes as ct
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5
FID32 = 1e-6

MODES_128 = [("none", 5), ("reference", 5), ("greedy", 2), ("greedy", 3), ("greedy", 4), ("greedy", 5),
             ("greedy", 6)]
MODES_64 = [("none", 5, True), ("reference", 5, True), ("greedy", 3, True), ("greedy", 4, True),
            ("greedy", 5, True), ("greedy", 5, False), ("greedy", 6, True)]


def gpu_run(n, ops, precision="c128", fusion="greedy", k=5, tc=True):
    import ket_b200 as kb
    from ket_b200 import _lib
    out = np.zeros(1 << n, dtype=np.complex128)
    opt = kb.make_options(precision, fusion, k, tc)
    _lib.check(_lib.lib.ketgpu_run(n, ops.ctypes.data, len(ops), ct.byref(opt), out.ctypes.data))
    return out


def fidelity(a, b):
    return abs(np.vdot(a, b)) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real)


def test_gate_battery_c128(golden):
    g = golden("gate_battery")
    for name, ops, want in zip(g["names"], g["ops"], g["states"]):
        for fusion, k in MODES_128:
            got = gpu_run(4, ops, "c128", fusion, k)
            assert np.abs(got - want).max() < TOL64, (name, fusion, k)


def test_gate_battery_c64(golden):
    g = golden("gate_battery")
    for name, ops, want in zip(g["names"], g["ops"], g["states"]):
        got = gpu_run(4, ops, "c64", "none")
        assert np.abs(got - want).max() < TOL32, name


@pytest.mark.parametrize("n", [6, 10, 12])
def test_random_mixed_c128_all_modes(golden, n):
    g = golden("random_mixed")
    want = g[f"state_{n}"]
    for fusion, k in MODES_128:
        got = gpu_run(n, g[f"ops_{n}"], "c128", fusion, k)
        assert np.abs(got - want).max() < TOL64, (fusion, k)


@pytest.mark.parametrize("n", [6, 10, 12])
def test_random_mixed_c64_all_modes(golden, n):
    g = golden("random_mixed")
    want = g[f"state_{n}"]
    for fusion, k, tc in MODES_64:
        got = gpu_run(n, g[f"ops_{n}"], "c64", fusion, k, tc)
        assert np.abs(got - want).max() < TOL32, (fusion, k, tc)
        assert fidelity(got, want) > 1 - FID32, (fusion, k, tc)


def _block_circuit(n, qubits, seed, depth=30):
    """A dense random block on `qubits` (one fused pass when k = len(qubits))."""
    from oracle.oracle import make_ops
    rng = np.random.default_rng(seed)
    gs = []
    for q in qubits:
        gs.append(("U", [q], rng.uniform(0, 2 * math.pi, 3).tolist()))
    for _ in range(depth):
        a, b = rng.choice(qubits, 2, replace=False).tolist()
        gs.append(("CX", [a, b]))
        gs.append(("U", [b], rng.uniform(0, 2 * math.pi, 3).tolist()))
        gs.append(("CP", [a, b], [float(rng.uniform(0, 6.28))]))
    return make_ops(gs)


# one target among qubits 0..5 with qubit 0 a group bit ("q1tgt5", "q2tgt5",
# "q3tgt4") takes the direct-store epilogue, like the blocks above qubit 4
TARGETS = {
    "low5": [0, 1, 2, 3, 4], "high5": None, "mixed5": [0, 3, 7, 11, 13], "spread5": [1, 5, 8, 12, 15],
    "q1tgt5": [1, 6, 9, 12, 14], "q2tgt5": [2, 7, 9, 11, 13],
    "low4": [0, 1, 2, 3], "mixed4": [2, 6, 9, 14], "high4": None, "q3tgt4": [3, 7, 10, 14],
    # k = 6: half-tile tensor copies (cp.async when qubit 0 is a target), two A regions, N = 128
    "low6": [0, 1, 2, 3, 4, 5], "high6": None, "mixed6": [0, 3, 7, 11, 13, 15],
    "spread6": [1, 5, 8, 12, 15, 17], "q1tgt6": [1, 6, 9, 12, 14, 15], "q2tgt6": [2, 7, 9, 11, 13, 15],
    "q2run6": [2, 3, 4, 5, 6, 7], "q6run6": [6, 7, 8, 9, 10, 11],
}


@pytest.mark.parametrize("name", sorted(TARGETS))
@pytest.mark.parametrize("n", [12, 16, 18])
def test_tensor_core_block_positions(oracle, name, n):
    """Single dense blocks on the tcgen05 path at every kind of target set."""
    import ket_b200 as kb
    k = int(name[-1])
    qs = TARGETS[name] or list(range(n - k, n))
    qs = [q for q in qs if q < n]
    if len(qs) != k or n < k + 7:
        pytest.skip("targets outside the register, or too few qubits for a 128-group tile")
    prep = _block_circuit(n, list(range(n)), seed=n, depth=2 * n)  # generic input state
    blk = _block_circuit(n, qs, seed=100 + n)
    ops = np.concatenate([prep, blk])
    want = oracle.run(n, ops, fuse=0)
    st = kb.plan_stats(kb.Circuit(n), None)  # warm import
    got = gpu_run(n, ops, "c64", "greedy", k, True)
    assert np.abs(got - want).max() < TOL32
    assert fidelity(got, want) > 1 - FID32
    # the block itself ran on the tensor cores
    from ket_b200 import _lib
    opt = kb.make_options("c64", "greedy", k, True)
    h = ct.c_void_p()
    _lib.check(_lib.lib.ketgpu_plan_create(n, blk.ctypes.data, len(blk), ct.byref(opt), ct.byref(h)))
    s = _lib.PlanStats()
    _lib.check(_lib.lib.ketgpu_plan_stats_get(h, ct.byref(s)))
    _lib.lib.ketgpu_plan_destroy(h)
    assert s.n_tensor >= 1


def test_brickwork_20q_d20_c128(oracle, golden):
    g = golden("brickwork_20q_d20")
    ops = g["ops"]
    want_full = oracle.run(20, ops, fuse=1)
    assert np.array_equal(want_full[:4096], g["head"])
    for fusion, k in [("none", 5), ("reference", 5), ("greedy", 5)]:
        got = gpu_run(20, ops, "c128", fusion, k)
        assert np.abs(got - want_full).max() < TOL64, fusion


def test_brickwork_20q_d20_c64(oracle, golden):
    g = golden("brickwork_20q_d20")
    ops = g["ops"]
    want = oracle.run(20, ops, fuse=1)
    for fusion, k, tc in [("none", 5, True), ("greedy", 5, True), ("greedy", 4, True), ("greedy", 5, False)]:
        got = gpu_run(20, ops, "c64", fusion, k, tc)
        assert np.abs(got - want).max() < TOL32, fusion
        assert fidelity(got, want) > 1 - FID32, fusion


def test_expval_matches_golden(golden):
    import ket_b200 as kb
    g = golden("expval")
    s = golden("random_mixed")["state_10"]
    for prec, tol in (("c128", 1e-12), ("c64", 1e-6)):
        d = kb.DeviceState(10, prec).from_numpy(s)
        for p, v in zip(g["paulis"], g["values"]):
            assert abs(d.expval(str(p)) - v) < tol, (prec, p)
        terms = list(zip(g["coeffs"].tolist(), [str(p) for p in g["paulis"]]))
        assert abs(d.expval(terms) - g["total"][0]) < 40 * tol
        d.close()


def test_expval_errors_like_ket():
    import ket_b200 as kb
    d = kb.DeviceState(2, "c128")
    with pytest.raises(ValueError):
        d.expval("Z")
    with pytest.raises(ValueError):
        d.expval("ZQ")
    assert abs(d.expval("ZZ") - 1.0) < 1e-15
    assert abs(d.expval("zi") - 1.0) < 1e-15


def test_norm_and_inner():
    import ket_b200 as kb
    from ket_b200.workloads import random_brickwork
    c = random_brickwork(16, 6, seed=3)
    a = kb.run_device(c, "c128")
    b = kb.run_device(c, "c128")
    assert abs(a.norm() - 1) < 1e-12
    assert abs(a.inner(b) - 1) < 1e-12


@pytest.mark.parametrize("k", [4, 5, 6])
def test_tensor_core_plans_keep_the_norm(k):
    """The norm capture / restore around tensor-core blocks: from a reset
    state (no capture pass: the norm is 1) and from an uploaded state of
    norm 4 (captured), the final norm equals the starting one, whether the
    restore sums the state itself or takes the last block's per-CTA sums;
    n from one tile (k + 7 qubits) up."""
    import ket_b200 as kb
    from ket_b200.workloads import random_brickwork
    for n in (k + 7, 16, 20):
        c = random_brickwork(n, 8, seed=n + k)
        opt = kb.make_options("c64", "greedy", k, True)
        plan = kb.Plan(n, c.to_ops(), opt)
        kinds = [plan.pass_info(i)["kind"] for i in range(int(plan.stats()["n_passes"]))]
        assert kinds[0] == 3 and kinds[-1] == 3  # NormCapture ... NormRestore
        plan.close()
        d = kb.run_device(c, options=opt)
        ref = kb.run_device(c, "c128")
        # bound: FP32 rounding of the rescaled amplitudes (~2^-24 / sqrt(2^n));
        # a CTA's partial missing from the sum would be off by 1/grid or more
        assert abs(d.norm() - 1.0) < 1e-7, (n, d.norm())
        assert fidelity(d.to_numpy(), ref.to_numpy()) > 1 - FID32
        # an uploaded state of norm 4 keeps its norm through the same circuit
        start = ref.to_numpy() * 2.0
        u = kb.DeviceState(n, "c64").from_numpy(start)
        u.apply(c, opt)
        assert abs(u.norm() / 4.0 - 1.0) < 1e-7, (n, u.norm())
        v = kb.DeviceState(n, "c128").from_numpy(start)
        v.apply(c, kb.make_options("c128", "greedy", 5, True))
        assert fidelity(u.to_numpy(), v.to_numpy()) > 1 - FID32
        for x in (d, ref, u, v):
            x.close()


def test_sampler_bit_exact_against_oracle(oracle, golden):
    import ket_b200 as kb
    s10 = golden("random_mixed")["state_10"]
    m = golden("measure")
    for prec in ("c128", "c64"):
        d = kb.DeviceState(10, prec).from_numpy(s10)
        host = d.to_numpy()
        for seed in (42, 7, 2024):
            u = m[f"uniforms_{seed}"]
            got = d.sample(u)
            want = oracle.sample_tree(10, host if prec == "c128" else host.astype(np.complex64), u)
            assert np.array_equal(got, want), (prec, seed)
            if prec == "c128":
                assert np.array_equal(got, m[f"outcomes_{seed}"])  # = ket::measure on this stream
        d.close()


@pytest.mark.parametrize("n", [5, 6, 11, 16, 20])
def test_sampler_tree_levels(oracle, n):
    import ket_b200 as kb
    from ket_b200.workloads import random_brickwork
    c = random_brickwork(n, 4, seed=n)
    d = kb.run_device(c, "c64")
    host = d.to_numpy().astype(np.complex64)
    u = kb.uniforms(99 + n, 20000)
    u = np.concatenate([u, [0.0, np.nextafter(1.0, 0.0), 0.5]])
    assert np.array_equal(d.sample(u), oracle.sample_tree(n, host, u))


def test_uniform_stream_is_std_mt19937(golden):
    import ket_b200 as kb
    from ket_b200.workloads import MT19937
    m = golden("measure")
    for seed in (42, 7, 2024):
        assert np.array_equal(kb.uniforms(seed, 2000), m[f"uniforms_{seed}"])
    r = MT19937(42)
    assert [r.canonical() for _ in range(5)] == list(m["uniforms_42"][:5])


def _diag_heavy(n, count, seed):
    """Random circuit dominated by diagonal gates (Z S Sdg T Tdg Rz CZ CP CRz)
    with some H, CX and U between them."""
    from oracle.oracle import make_ops
    rng = np.random.default_rng(seed)
    diag1 = ["Z", "S", "Sdg", "T", "Tdg", "Rz"]
    diag2 = ["CZ", "CP", "CRz"]
    gs = [("H", [q]) for q in range(n)]
    for _ in range(count):
        r = rng.random()
        if r < 0.35:
            g = diag1[int(rng.integers(len(diag1)))]
            gs.append((g, [int(rng.integers(n))], [float(rng.uniform(0, 2 * math.pi))] if g == "Rz" else []))
        elif r < 0.8:
            g = diag2[int(rng.integers(len(diag2)))]
            a, b = (int(x) for x in rng.choice(n, 2, replace=False))
            gs.append((g, [a, b], [float(rng.uniform(0, 2 * math.pi))] if g != "CZ" else []))
        elif r < 0.9:
            a, b = (int(x) for x in rng.choice(n, 2, replace=False))
            gs.append(("CX", [a, b]))
        else:
            gs.append(("U", [int(rng.integers(n))], rng.uniform(0, 2 * math.pi, 3).tolist()))
    return make_ops(gs)


@pytest.mark.parametrize("n", [5, 6, 7, 12, 13, 15])
def test_diagonal_runs_qft_pattern(oracle, n):
    """H on all, CP(pi/2^(j-i)) on every pair, GHZ ladder, Rz layer: the CP
    run becomes one diagonal pass (low-bit table + per-chunk tables)."""
    from ket_b200.workloads import qft_ghz_rz
    ops = qft_ghz_rz(n).to_ops()
    want = oracle.run(n, ops, fuse=0)
    for k in (3, 5):
        got = gpu_run(n, ops, "c128", "greedy", k)
        assert np.abs(got - want).max() < TOL64, k
    got = gpu_run(n, ops, "c64", "greedy", 5, True)
    assert np.abs(got - want).max() < TOL32
    assert fidelity(got, want) > 1 - FID32


@pytest.mark.parametrize("n,seed", [(9, 1), (14, 2), (16, 3)])
def test_diagonal_heavy_random(oracle, n, seed):
    ops = _diag_heavy(n, 300, seed)
    want = oracle.run(n, ops, fuse=0)
    for fusion, k in [("greedy", 3), ("greedy", 5), ("greedy", 6), ("learned", 5)]:
        got = gpu_run(n, ops, "c128", fusion, k)
        assert np.abs(got - want).max() < TOL64, (fusion, k)
    for tc in (True, False):
        got = gpu_run(n, ops, "c64", "greedy", 5, tc)
        assert np.abs(got - want).max() < TOL32
        assert fidelity(got, want) > 1 - FID32


@pytest.mark.parametrize("qs", [[0, 1], [3, 9], [1, 2, 3], [0, 7, 12]])
def test_small_blocks_padded_onto_the_tensor_cores(oracle, qs):
    """2- and 3-qubit dense blocks in complex64 run as 4-qubit tensor-core
    blocks (identity on the padding qubits)."""
    import ket_b200 as kb
    from ket_b200 import _lib
    n = 14
    prep = _block_circuit(n, list(range(n)), seed=5, depth=2 * n)
    blk = _block_circuit(n, qs, seed=17)
    ops = np.concatenate([prep, blk])
    want = oracle.run(n, ops, fuse=0)
    got = gpu_run(n, ops, "c64", "greedy", len(qs), True)
    assert np.abs(got - want).max() < TOL32
    assert fidelity(got, want) > 1 - FID32
    opt = kb.make_options("c64", "greedy", len(qs), True)
    h = ct.c_void_p()
    _lib.check(_lib.lib.ketgpu_plan_create(n, blk.ctypes.data, len(blk), ct.byref(opt), ct.byref(h)))
    ks = []
    for i in range(int(kb.plan_stats(type("C", (), {"to_ops": lambda s: blk, "n_qubits": n})(), opt)["n_passes"])):
        kind, k, tc, b = ct.c_int32(), ct.c_int32(), ct.c_int32(), ct.c_double()
        _lib.check(_lib.lib.ketgpu_plan_pass_info(h, i, ct.byref(kind), ct.byref(k), ct.byref(tc), ct.byref(b)))
        if kind.value == 2:
            ks.append((k.value, tc.value))
    _lib.lib.ketgpu_plan_destroy(h)
    assert ks and all(x == (4, 1) for x in ks)
