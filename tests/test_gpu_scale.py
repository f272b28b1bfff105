"""The sampling and adjoint workloads at their own sizes, against the CPU
oracle.

* Sampling: the QFT-pattern + GHZ + Rz circuit at 30 qubits in complex64
  (8 GiB state), 10^6 draws of uniform_real_distribution<double>(0, 1) on
  std::mt19937{42}; every drawn index bit-exact against the oracle's
  fixed-tree sampler over the downloaded state (ko_sample_tree, the
  restatement of src/measurement.cpp:12-21 that shares the GPU's summation
  tree).
* Adjoint: the 24-qubit, 8-layer Ry/Rz + CX-ring ansatz (384 parameters), 64
  random Pauli strings, a batch of 64 parameter sets, complex64 states with
  checkpoints every 2 layers, through the torch.autograd.Function.  Two sets
  are checked against the FP64 oracle adjoint (1e-5, the complex64 bar) and
  six gradients against central differences (h = 1e-3) of the complex128
  forward, whose states the other tests pin to ket::run at 1e-12.
"""
import math
import multiprocessing as mp
from concurrent.futures import ProcessPoolExecutor

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_sampling_30q_bit_exact_against_oracle(oracle):
    import ket_b200 as ket
    from ket_b200.workloads import qft_ghz_rz
    n, shots = 30, 10 ** 6
    d = ket.run_device(qft_ghz_rz(n, seed=7), options=ket.make_options("c64", "greedy", 5, True))
    u = ket.uniforms(42, shots)
    got = d.sample(u)
    host = d.to_numpy_raw()
    norm = d.norm()
    d.close()
    assert abs(norm - 1.0) < 1e-5
    want = oracle.sample_tree(n, host, u)
    assert np.array_equal(got, want)
    vals, counts = np.unique(got, return_counts=True)
    assert counts.sum() == shots and len(vals) > 1000


def _oracle_adjoint(args):
    """One FP64 adjoint on the CPU (runs in a spawned worker)."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from oracle.oracle import Oracle
    n, ops, pidx, theta, ham = args
    return Oracle().adjoint(n, ops, pidx, theta, ham)


def test_adjoint_24q_batch64_against_fp64_oracle_and_finite_differences():
    import torch

    import ket_b200 as ket
    from ket_b200.autograd import adjoint_expval_torch
    from ket_b200.workloads import random_pauli_sum, variational_ansatz
    n, layers, batch = 24, 8, 64
    circ, pidx = variational_ansatz(n, layers)
    npar = int((pidx >= 0).sum())
    assert npar == 384
    ham = random_pauli_sum(n, 64, seed=11)
    theta_np = np.random.default_rng(12).uniform(-math.pi, math.pi, (batch, npar))
    ops = circ.to_ops()
    checked = (0, 37)
    # the FP64 oracle (minutes of CPU per set) runs in spawned workers
    # while the GPU works
    pool = ProcessPoolExecutor(max_workers=len(checked), mp_context=mp.get_context("spawn"))
    futs = [pool.submit(_oracle_adjoint, (n, ops, pidx, theta_np[b], ham)) for b in checked]

    theta = torch.tensor(theta_np, dtype=torch.float64, requires_grad=True)
    vals = adjoint_expval_torch(theta, circ, pidx, ham, "c64", 2)
    vals.sum().backward()
    grads = theta.grad.numpy()
    values = vals.detach().numpy()
    assert np.all(np.isfinite(grads)) and np.abs(grads).max() > 1e-3

    h = 1e-3
    ks = np.random.default_rng(13).choice(npar, 6, replace=False)
    for k in ks:
        f = []
        for sgn in (1, -1):
            th = theta_np[1].copy()
            th[k] += sgn * h
            o = ops.copy()
            for i, p in enumerate(pidx):
                if p >= 0:
                    o[i]["p"][0] = th[p]
            d = ket.DeviceState(n, "c128")
            d.apply(o, ket.make_options("c128", "greedy", 5, True))
            f.append(d.expval(ham))
            d.close()
        assert abs((f[0] - f[1]) / (2 * h) - grads[1][k]) < 1e-5

    for b, fut in zip(checked, futs):
        v, g = fut.result(timeout=1500)
        assert abs(values[b] - v) < 1e-5
        assert np.abs(grads[b] - g).max() < 1e-5
    pool.shutdown()
