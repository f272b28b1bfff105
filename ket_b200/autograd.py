"""Adjoint gradients of Pauli-sum expectations, and their torch.autograd
wrapper.

``adjoint_expval`` evaluates <psi(theta)|H|psi(theta)> and its full gradient
for a batch of parameter sets with one reverse sweep each
(ketgpu_adjoint).  ``AdjointExpval`` exposes it to torch: the forward pass
returns the batch of expectations and keeps the gradients, the backward
pass scales them by the incoming gradient.  torch is only the autograd
plumbing here; the state vectors and sweeps live in libket_b200.so.
"""
from __future__ import annotations

import ctypes as ct
from typing import Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import check, lib
from .circuit import Circuit


def adjoint_expval(circuit: Circuit, param_index: np.ndarray, params: np.ndarray,
                   hamiltonian: Sequence[Tuple[float, str]], precision: str = "c64",
                   checkpoint_every: int = 2, method: str = "auto") -> Tuple[np.ndarray, np.ndarray]:
    """values (batch,), grads (batch, n_params) for params of shape (batch, n_params).

    method: "auto", "per_gate", "tiled" or "tiled_jit" (the sweep kernels;
    same results up to rounding)."""
    ops = circuit.to_ops()
    pidx = np.ascontiguousarray(param_index, dtype=np.int32)
    if len(pidx) != len(ops):
        raise ValueError("param_index must have one entry per op")
    prm = np.ascontiguousarray(np.atleast_2d(params), dtype=np.float64)
    batch, npar = prm.shape
    coeffs = np.array([c for c, _ in hamiltonian], dtype=np.float64)
    arr, keep = _lib.c_strings([p for _, p in hamiltonian])
    values = np.zeros(batch, dtype=np.float64)
    grads = np.zeros((batch, npar), dtype=np.float64)
    prec = {"c64": _lib.C64, "c128": _lib.C128}[precision]
    meth = {"auto": 0, "per_gate": 1, "tiled": 2, "tiled_jit": 3}[method]
    check(lib.ketgpu_adjoint_ex(circuit.n_qubits, ops.ctypes.data, len(ops), pidx.ctypes.data, prm.ctypes.data,
                                npar, batch, coeffs.ctypes.data, ct.cast(arr, ct.c_void_p), len(hamiltonian),
                                prec, int(checkpoint_every), meth, values.ctypes.data, grads.ctypes.data))
    return values, grads


def jit_info() -> dict:
    """Per-block compiled adjoint kernels: NVRTC availability, kernels cached
    and launches so far."""
    a = ct.c_int32()
    k = ct.c_uint64()
    n = ct.c_uint64()
    check(lib.ketgpu_adjoint_jit_info(ct.byref(a), ct.byref(k), ct.byref(n)))
    return {"available": bool(a.value), "kernels": k.value, "launches": n.value}


def _function():
    import torch

    class AdjointExpval(torch.autograd.Function):
        """f(theta) = <psi(theta)|H|psi(theta)> for each row of theta."""

        @staticmethod
        def forward(ctx, theta, circuit, param_index, hamiltonian, precision="c64", checkpoint_every=2):
            t = theta.detach()
            values, grads = adjoint_expval(circuit, param_index, t.to("cpu", torch.float64).numpy(),
                                           hamiltonian, precision, checkpoint_every)
            g = torch.from_numpy(grads).to(device=theta.device, dtype=theta.dtype)
            ctx.save_for_backward(g)
            out = torch.from_numpy(values).to(device=theta.device, dtype=theta.dtype)
            return out if theta.dim() == 2 else out[0]

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            go = grad_out.reshape(-1, 1) if grad_out.dim() else grad_out.reshape(1, 1)
            grad = go * g
            return (grad if grad_out.dim() else grad[0]), None, None, None, None, None

    return AdjointExpval


class _Lazy:
    fn = None


def adjoint_expval_torch(theta, circuit, param_index, hamiltonian, precision="c64", checkpoint_every=2):
    """torch entry point: differentiable w.r.t. theta ((batch, P) or (P,))."""
    if _Lazy.fn is None:
        _Lazy.fn = _function()
    return _Lazy.fn.apply(theta, circuit, param_index, hamiltonian, precision, checkpoint_every)
