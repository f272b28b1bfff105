"""Adjoint gradients on the GPU against the FP64 CPU adjoint (oracle),
central finite differences, and the torch autograd wrapper.

Tolerances: complex128 mode 1e-9 absolute on values and gradients against
the FP64 oracle; complex64 mode 1e-5 (the north-star bar for FP32 states
with FP64 accumulation); finite differences (h = 1e-3, error O(h^2)) 5e-6.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _random_param_circuit(n, count, seed):
    import ket_b200 as ket
    rng = np.random.default_rng(seed)
    c = ket.Circuit(n)
    pidx = []
    k = 0
    for _ in range(count):
        kind = rng.integers(0, 10)
        a, b = (int(x) for x in rng.choice(n, 2, replace=False))
        if kind < 3:
            getattr(c, ["rx", "ry", "rz"][kind])(a, 0.0)
            pidx.append(k)
            k += 1
        elif kind < 6:
            getattr(c, ["crx", "cry", "crz"][kind - 3])(a, b, 0.0)
            pidx.append(k)
            k += 1
        elif kind == 6:
            c.cp(a, b, 0.0)
            pidx.append(k)
            k += 1
        elif kind == 7:
            c.cx(a, b)
            pidx.append(-1)
        elif kind == 8:
            c.h(a)
            pidx.append(-1)
        else:
            c.u(a, *rng.uniform(0, 6.28, 3))
            pidx.append(-1)
    return c, np.array(pidx, dtype=np.int32), k


def _with_params(circ, pidx, theta):
    ops = circ.to_ops().copy()
    for i, p in enumerate(pidx):
        if p >= 0:
            ops[i]["p"][0] = theta[p]
    return ops


@pytest.mark.parametrize("prec,tol", [("c128", 1e-9), ("c64", 1e-5)])
def test_adjoint_matches_fp64_oracle(oracle, prec, tol):
    from ket_b200.autograd import adjoint_expval
    from ket_b200.workloads import random_pauli_sum
    n = 7
    circ, pidx, npar = _random_param_circuit(n, 60, seed=1)
    ham = random_pauli_sum(n, 12, seed=2)
    rng = np.random.default_rng(3)
    thetas = rng.uniform(-math.pi, math.pi, (4, npar))
    vals, grads = adjoint_expval(circ, pidx, thetas, ham, prec, checkpoint_every=0)
    for b in range(4):
        v, g = oracle.adjoint(n, circ.to_ops(), pidx, thetas[b], ham)
        assert abs(vals[b] - v) < tol
        assert np.abs(grads[b] - g).max() < tol


@pytest.mark.parametrize("ckpt", [0, 1, 2])
def test_ansatz_checkpointing_and_finite_differences(oracle, ckpt):
    from ket_b200.autograd import adjoint_expval
    from ket_b200.workloads import random_pauli_sum, variational_ansatz
    n, layers = 8, 4
    circ, pidx = variational_ansatz(n, layers)
    npar = int((pidx >= 0).sum())
    ham = random_pauli_sum(n, 16, seed=5)
    theta = np.random.default_rng(6).uniform(-math.pi, math.pi, (2, npar))
    vals, grads = adjoint_expval(circ, pidx, theta, ham, "c128", checkpoint_every=ckpt)
    v0, g0 = oracle.adjoint(n, circ.to_ops(), pidx, theta[0], ham)
    assert abs(vals[0] - v0) < 1e-10 and np.abs(grads[0] - g0).max() < 1e-10
    h = 1e-3
    for k in (0, 7, npar // 2, npar - 1):
        e = np.zeros(npar)
        e[k] = h
        fp = oracle.expval_sum(n, oracle.run(n, _with_params(circ, pidx, theta[1] + e), fuse=0), ham)
        fm = oracle.expval_sum(n, oracle.run(n, _with_params(circ, pidx, theta[1] - e), fuse=0), ham)
        assert abs((fp - fm) / (2 * h) - grads[1][k]) < 5e-6


def test_c64_adjoint_within_1e5_of_fp64_at_scale():
    """The 24-qubit ansatz shape at 14 qubits, 8 layers, 64 Pauli terms."""
    from ket_b200.autograd import adjoint_expval
    from ket_b200.workloads import random_pauli_sum, variational_ansatz
    n = 14
    circ, pidx = variational_ansatz(n, 8)
    npar = int((pidx >= 0).sum())
    ham = random_pauli_sum(n, 64, seed=7)
    theta = np.random.default_rng(8).uniform(-math.pi, math.pi, (3, npar))
    v64, g64 = adjoint_expval(circ, pidx, theta, ham, "c64", checkpoint_every=2)
    v128, g128 = adjoint_expval(circ, pidx, theta, ham, "c128", checkpoint_every=2)
    assert np.abs(v64 - v128).max() < 1e-5
    assert np.abs(g64 - g128).max() < 1e-5


def test_torch_autograd_function():
    import torch

    from ket_b200.autograd import adjoint_expval, adjoint_expval_torch
    from ket_b200.workloads import random_pauli_sum, variational_ansatz
    n = 6
    circ, pidx = variational_ansatz(n, 2)
    npar = int((pidx >= 0).sum())
    ham = random_pauli_sum(n, 8, seed=9)
    theta = torch.tensor(np.random.default_rng(10).uniform(-3, 3, (3, npar)), dtype=torch.float64,
                         requires_grad=True)
    out = adjoint_expval_torch(theta, circ, pidx, ham, "c128", 1)
    w = torch.tensor([0.5, -1.0, 2.0], dtype=torch.float64)
    (out * w).sum().backward()
    vals, grads = adjoint_expval(circ, pidx, theta.detach().numpy(), ham, "c128", 1)
    assert np.allclose(out.detach().numpy(), vals, atol=1e-12)
    assert np.allclose(theta.grad.numpy(), w.numpy()[:, None] * grads, atol=1e-12)


def test_adjoint_errors():
    from ket_b200.autograd import adjoint_expval
    import ket_b200 as ket
    c = ket.Circuit(3)
    c.h(0)
    c.cx(0, 1)
    with pytest.raises(ValueError):  # a non-rotation marked as parameterised
        adjoint_expval(c, np.array([0, -1], dtype=np.int32), np.zeros((1, 1)), [(1.0, "ZZZ")], "c128")
    c2 = ket.Circuit(3)
    c2.ry(0, 0.0)
    with pytest.raises(ValueError):  # bad Pauli string
        adjoint_expval(c2, np.array([0], dtype=np.int32), np.zeros((1, 1)), [(1.0, "ZZ")], "c128")


def _mixed_circuit(n, count, seed, barriers=3):
    """Every gate kind ket has, with barriers; the rotations are parameters."""
    from oracle.oracle import ARITY, GATES, NPARAMS, make_ops
    rng = np.random.default_rng(seed)
    gs, pidx = [], []
    k = 0
    pool = [g for g in GATES if ARITY[g] >= 1]
    step = count // barriers + 1
    for i in range(count):
        if barriers and i % step == step - 1:
            gs.append(("Barrier", []))
            pidx.append(-1)
            continue
        g = pool[int(rng.integers(len(pool)))]
        qs = [int(x) for x in rng.choice(n, ARITY[g], replace=False)]
        ps = [float(x) for x in rng.uniform(0, 2 * math.pi, NPARAMS.get(g, 0))]
        gs.append((g, qs, ps))
        pidx.append(k if g in ("Rx", "Ry", "Rz", "CRx", "CRy", "CRz", "CP") else -1)
        k += pidx[-1] >= 0
    return make_ops(gs), np.array(pidx, dtype=np.int32), k


class _OpsCircuit:
    """Minimal circuit wrapper for adjoint_expval over a raw op array."""

    def __init__(self, n, ops):
        self.n_qubits = n
        self._ops = ops

    def to_ops(self):
        return self._ops


@pytest.mark.parametrize("prec,n,tol", [("c128", 11, 1e-9), ("c128", 13, 1e-9), ("c64", 12, 1e-5),
                                        ("c64", 14, 1e-5)])
@pytest.mark.parametrize("ckpt", [0, 1])
def test_tiled_sweep_matches_fp64_oracle(oracle, prec, n, tol, ckpt):
    """The tiled sweeps (blocks of gates in shared memory) against the FP64
    oracle adjoint, over every gate kind, with barriers and checkpoints."""
    from ket_b200.autograd import adjoint_expval
    from ket_b200.workloads import random_pauli_sum
    ops, pidx, npar = _mixed_circuit(n, 120, seed=n + 7 * ckpt)
    circ = _OpsCircuit(n, ops)
    ham = random_pauli_sum(n, 10, seed=n)
    thetas = np.random.default_rng(n + 1).uniform(-math.pi, math.pi, (3, npar))
    vals, grads = adjoint_expval(circ, pidx, thetas, ham, prec, checkpoint_every=ckpt, method="tiled")
    for b in range(3):
        v, g = oracle.adjoint(n, ops, pidx, thetas[b], ham)
        assert abs(vals[b] - v) < tol
        assert np.abs(grads[b] - g).max() < tol


@pytest.mark.parametrize("prec,tol", [("c128", 1e-10), ("c64", 2e-5)])
def test_tiled_and_per_gate_sweeps_agree(prec, tol):
    """The 24-qubit ansatz shape at 15 qubits: both sweep methods."""
    from ket_b200.autograd import adjoint_expval
    from ket_b200.workloads import random_pauli_sum, variational_ansatz
    n = 15
    circ, pidx = variational_ansatz(n, 6)
    npar = int((pidx >= 0).sum())
    ham = random_pauli_sum(n, 32, seed=21)
    theta = np.random.default_rng(22).uniform(-math.pi, math.pi, (5, npar))
    v1, g1 = adjoint_expval(circ, pidx, theta, ham, prec, checkpoint_every=2, method="per_gate")
    v2, g2 = adjoint_expval(circ, pidx, theta, ham, prec, checkpoint_every=2, method="tiled")
    assert np.abs(v1 - v2).max() < tol
    assert np.abs(g1 - g2).max() < tol


def test_tiled_sweep_needs_a_full_tile():
    from ket_b200.autograd import adjoint_expval
    from ket_b200.workloads import variational_ansatz
    circ, pidx = variational_ansatz(10, 1)
    npar = int((pidx >= 0).sum())
    with pytest.raises(ValueError):
        adjoint_expval(circ, pidx, np.zeros((1, npar)), [(1.0, "Z" * 10)], "c64", method="tiled")


def test_hamiltonian_with_more_terms_than_shared_memory_holds(oracle):
    """1100 Pauli terms: lambda = H psi takes the global-memory form (the
    shared-memory form holds 1024 terms)."""
    from ket_b200.autograd import adjoint_expval
    from ket_b200.workloads import random_pauli_sum, variational_ansatz
    n = 12
    circ, pidx = variational_ansatz(n, 2)
    npar = int((pidx >= 0).sum())
    ham = random_pauli_sum(n, 1100, seed=31)
    theta = np.random.default_rng(32).uniform(-math.pi, math.pi, (1, npar))
    vals, grads = adjoint_expval(circ, pidx, theta, ham, "c128", checkpoint_every=1)
    v, g = oracle.adjoint(n, circ.to_ops(), pidx, theta[0], ham)
    assert abs(vals[0] - v) < 1e-9
    assert np.abs(grads[0] - g).max() < 1e-9


@pytest.mark.parametrize("n", [12, 14])
def test_per_block_compiled_sweeps_match_fp64_oracle(oracle, n):
    """The per-block kernels generated and compiled at run time (NVRTC), over
    every gate kind with barriers and checkpoints, against the FP64 oracle
    and the compiled sweep."""
    from ket_b200.autograd import adjoint_expval, jit_info
    from ket_b200.workloads import random_pauli_sum
    info0 = jit_info()
    ops, pidx, npar = _mixed_circuit(n, 90, seed=40 + n)
    circ = _OpsCircuit(n, ops)
    ham = random_pauli_sum(n, 10, seed=n + 3)
    thetas = np.random.default_rng(n + 4).uniform(-math.pi, math.pi, (2, npar))
    vj, gj = adjoint_expval(circ, pidx, thetas, ham, "c64", checkpoint_every=1, method="tiled_jit")
    vt, gt = adjoint_expval(circ, pidx, thetas, ham, "c64", checkpoint_every=1, method="tiled")
    for b in range(2):
        v, g = oracle.adjoint(n, ops, pidx, thetas[b], ham)
        assert abs(vj[b] - v) < 1e-5
        assert np.abs(gj[b] - g).max() < 1e-5
    assert np.abs(gj - gt).max() < 2e-5
    info = jit_info()
    assert info["available"], "NVRTC is part of the CUDA toolkit on a B200 box; the compiled sweeps must run"
    assert info["launches"] > info0["launches"]


def test_per_block_compiled_sweeps_on_the_ansatz():
    from ket_b200.autograd import adjoint_expval, jit_info
    from ket_b200.workloads import random_pauli_sum, variational_ansatz
    n = 16
    circ, pidx = variational_ansatz(n, 4)
    npar = int((pidx >= 0).sum())
    ham = random_pauli_sum(n, 16, seed=41)
    theta = np.random.default_rng(42).uniform(-math.pi, math.pi, (3, npar))
    v1, g1 = adjoint_expval(circ, pidx, theta, ham, "c64", checkpoint_every=2, method="tiled")
    v2, g2 = adjoint_expval(circ, pidx, theta, ham, "c64", checkpoint_every=2, method="auto")
    v3, g3 = adjoint_expval(circ, pidx, theta, ham, "c128", checkpoint_every=2, method="per_gate")
    assert np.abs(v2 - v3).max() < 1e-5 and np.abs(g2 - g3).max() < 1e-5
    assert np.abs(g1 - g2).max() < 2e-5
    # the layers repeat: one compiled kernel per distinct block structure
    info = jit_info()
    assert info["available"]
    assert 0 < info["kernels"] <= 64
