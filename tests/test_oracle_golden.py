"""The CPU oracle pinned against ket's own outputs (tests/golden, made by
tests/golden/make_golden.py from ket::run / expval / measure / sample)."""
import numpy as np

from oracle.oracle import CODE, make_ops


def test_gate_battery_bit_exact(oracle, golden):
    g = golden("gate_battery")
    for name, ops, want in zip(g["names"], g["ops"], g["states"]):
        got = oracle.run(4, ops, fuse=1)
        assert np.array_equal(got, want), name


def test_random_mixed_bit_exact_with_reference_fuser(oracle, golden):
    g = golden("random_mixed")
    for n in (6, 10, 12):
        got = oracle.run(n, g[f"ops_{n}"], fuse=1)
        assert np.array_equal(got, g[f"state_{n}"]), n
        # unfused differs from ket's fused run only by rounding
        un = oracle.run(n, g[f"ops_{n}"], fuse=0)
        assert np.abs(un - g[f"state_{n}"]).max() < 1e-12


def test_brickwork_20q(oracle, golden):
    g = golden("brickwork_20q_d20")
    st = oracle.run(20, g["ops"], fuse=1)
    assert np.array_equal(st[:4096], g["head"])
    assert np.array_equal(st[g["idx"]], g["sampled"])
    assert abs(np.vdot(st, st).real - g["norm"][0]) < 1e-12


def test_expval(oracle, golden):
    g = golden("expval")
    s = golden("random_mixed")["state_10"]
    for p, v in zip(g["paulis"], g["values"]):
        assert oracle.expval(10, s, str(p)) == v
    terms = list(zip(g["coeffs"].tolist(), [str(p) for p in g["paulis"]]))
    assert oracle.expval_sum(10, s, terms) == g["total"][0]


def test_expval_errors(oracle):
    s = np.zeros(4, dtype=np.complex128)
    s[0] = 1
    import pytest
    with pytest.raises(ValueError):
        oracle.expval(2, s, "Z")        # length mismatch (observable.cpp:63-66)
    with pytest.raises(ValueError):
        oracle.expval(2, s, "ZQ")       # bad character (observable.cpp:94-96)


def test_measure_stream_and_sequential(oracle, golden):
    g = golden("measure")
    s = golden("random_mixed")["state_10"]
    for seed in (42, 7, 2024):
        u = oracle.uniforms(seed, 2000)
        assert np.array_equal(u, g[f"uniforms_{seed}"])
        assert np.array_equal(oracle.measure_sequential(10, s, u), g[f"outcomes_{seed}"])
        # the fixed-tree sampler agrees with ket's sequential scan on these draws
        assert np.array_equal(oracle.sample_tree(10, s, u), g[f"outcomes_{seed}"])


def test_tree_sampler_equals_sequential_when_single_segment(oracle):
    rng = np.random.default_rng(3)
    for n in range(0, 6):
        s = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
        s /= np.linalg.norm(s)
        u = np.concatenate([rng.random(500), [0.0, np.nextafter(1.0, 0.0)]])
        assert np.array_equal(oracle.sample_tree(n, s, u), oracle.measure_sequential(n, s, u))


def test_tree_sampler_edge_cases(oracle):
    # zero-probability tail: draws beyond the total mass return the last index
    s = np.zeros(1 << 8, dtype=np.complex128)
    s[3] = 0.5
    out = oracle.sample_tree(8, s, np.array([0.1, 0.2499, 0.9]))
    assert list(out) == [3, 3, 255]
    assert list(oracle.measure_sequential(8, s, np.array([0.1, 0.2499, 0.9]))) == [3, 3, 255]


def test_block_matrix_matches_sequential_application(oracle):
    rng = np.random.default_rng(4)
    gates = [("H", [2]), ("CX", [2, 5]), ("Rz", [5], [0.4]), ("CP", [5, 2], [1.3]), ("U", [2], [0.1, 0.2, 0.3])]
    ops = make_ops(gates)
    m = oracle.block_matrix(ops, [2, 5])
    n = 7
    s = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    a = oracle.apply(n, s, ops, fuse=0)
    b = oracle.apply_matrix(n, s, [2, 5], m)
    assert np.abs(a - b).max() < 1e-13


def test_adjoint_oracle_against_finite_differences(oracle):
    ops = make_ops([("Ry", [0], [0.0]), ("Rz", [1], [0.0]), ("CX", [0, 1]), ("Rx", [2], [0.0]),
                    ("CRy", [2, 0], [0.0]), ("CP", [1, 2], [0.0]), ("Rz", [0], [0.0])])
    pidx = np.array([0, 1, -1, 2, 3, 4, 5], dtype=np.int32)
    params = np.array([0.3, -1.2, 0.8, 2.1, -0.4, 1.7])
    terms = [(0.7, "ZXY"), (-1.3, "IZZ"), (0.4, "XIX")]

    def value(p):
        o = ops.copy()
        for i, k in enumerate(pidx):
            if k >= 0:
                o[i]["p"][0] = p[k]
        st = oracle.run(3, o, fuse=0)
        return oracle.expval_sum(3, st, terms)

    v, grad = oracle.adjoint(3, ops, pidx, params, terms)
    assert abs(v - value(params)) < 1e-12
    h = 1e-5
    for k in range(len(params)):
        e = np.zeros_like(params)
        e[k] = h
        fd = (value(params + e) - value(params - e)) / (2 * h)
        assert abs(fd - grad[k]) < 1e-8, k


def test_mlp_oracle_gradients_match_finite_differences(oracle):
    rng = np.random.default_rng(0)
    w = [rng.standard_normal((128, 48)).astype(np.float32) * 0.1, rng.standard_normal(128).astype(np.float32) * 0.1,
         rng.standard_normal((128, 128)).astype(np.float32) * 0.1, rng.standard_normal(128).astype(np.float32) * 0.1,
         rng.standard_normal(128).astype(np.float32) * 0.1, np.array([0.05], dtype=np.float32)]
    x = rng.standard_normal((8, 48)).astype(np.float32)
    y = rng.standard_normal(8).astype(np.float32)
    loss, grads = oracle.mlp_backward(w, x, y)
    out = oracle.mlp_forward(w, x)
    assert abs(loss - np.mean((out - y) ** 2)) < 1e-9
    # spot-check a few weights by central differences in double
    for (wi, idx) in [(0, (3, 7)), (2, (10, 20)), (4, (5,)), (5, (0,))]:
        h = 1e-2
        wp = [a.astype(np.float64).copy() for a in w]
        wm = [a.astype(np.float64).copy() for a in w]
        wp[wi][idx] += h
        wm[wi][idx] -= h
        fp = np.mean((oracle.mlp_forward([a.astype(np.float32) for a in wp], x) - y) ** 2)
        fm = np.mean((oracle.mlp_forward([a.astype(np.float32) for a in wm], x) - y) ** 2)
        # float32 weights: perturbation is exact at h=1e-2 only to ~1e-7 relative
        assert abs((fp - fm) / (2 * h) - grads[wi][idx]) < 1e-3


def test_op_codes_match_ket_gate_numbering():
    assert CODE["H"] == 0 and CODE["U"] == 11 and CODE["CH"] == 12 and CODE["Swap"] == 21
    assert CODE["CSwap"] == 23 and CODE["Probe"] == 27
