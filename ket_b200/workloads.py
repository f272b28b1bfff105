"""Seeded synthetic circuits of the benchmark shapes.

* ``random_brickwork(n, depth, seed)`` -- every layer applies U(theta, phi,
  lambda) to every qubit, angles uniform on [0, 2pi), then CX on the
  nearest-neighbour brick wall (pairs (0,1),(2,3),... on even layers,
  (1,2),(3,4),... on odd layers).  20q x 20 and 30q x 40 are the headline
  shapes.  Angles are the draws of uniform_real_distribution<double>(0, 2pi)
  on std::mt19937{seed}, three per qubit per layer, in (layer, qubit,
  theta/phi/lambda) order, so a C++ harness reproduces the same circuit.
* ``qft_ghz_rz(n, seed)`` -- H on every qubit, CP(pi/2^(j-i)) for all i<j,
  a GHZ ladder (H q0, CX q_i -> q_i+1) and a final Rz layer.
* ``variational_ansatz(n, layers)`` -- Ry then Rz on every qubit, then a CX
  ring, per layer; returns the ops and the parameter index of every angle.
* ``random_pauli_sum(n, terms, seed)`` -- strings uniform over IXYZ with
  N(0,1) coefficients.
* ``random_mixed(n, depth, seed)`` -- layers drawn from the gate mix
  H/S/T/Rx/Ry/Rz/U/CX/CZ/CP/CRz/SWAP/CCX/CSWAP with random targets.
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

from .circuit import Circuit

TWO_PI = 6.283185307179586


class MT19937:
    """std::mt19937 with libstdc++'s generate_canonical<double, 53>."""

    def __init__(self, seed: int):
        mt = [0] * 624
        mt[0] = seed & 0xFFFFFFFF
        for i in range(1, 624):
            mt[i] = (1812433253 * (mt[i - 1] ^ (mt[i - 1] >> 30)) + i) & 0xFFFFFFFF
        self.mt, self.idx = mt, 624

    def _next(self) -> int:
        if self.idx >= 624:
            mt = self.mt
            for i in range(624):
                y = (mt[i] & 0x80000000) | (mt[(i + 1) % 624] & 0x7FFFFFFF)
                mt[i] = mt[(i + 397) % 624] ^ (y >> 1) ^ (0x9908B0DF if y & 1 else 0)
            self.idx = 0
        y = self.mt[self.idx]
        self.idx += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        return y & 0xFFFFFFFF

    def canonical(self) -> float:
        lo = float(self._next())
        hi = float(self._next())
        r = (lo + hi * 4294967296.0) / 18446744073709551616.0
        return r if r < 1.0 else math.nextafter(1.0, 0.0)

    def uniform(self, a: float, b: float) -> float:
        return self.canonical() * (b - a) + a


def random_brickwork(n: int, depth: int, seed: int = 1234) -> Circuit:
    rng = MT19937(seed)
    c = Circuit(n)
    for layer in range(depth):
        for q in range(n):
            th, ph, la = rng.uniform(0.0, TWO_PI), rng.uniform(0.0, TWO_PI), rng.uniform(0.0, TWO_PI)
            c.u(q, th, ph, la)
        for a in range(layer % 2, n - 1, 2):
            c.cx(a, a + 1)
    return c


def qft_ghz_rz(n: int, seed: int = 7) -> Circuit:
    rng = MT19937(seed)
    c = Circuit(n)
    for q in range(n):
        c.h(q)
    for i in range(n):
        for j in range(i + 1, n):
            c.cp(i, j, math.pi / (2 ** (j - i)))
    c.h(0)
    for i in range(n - 1):
        c.cx(i, i + 1)
    for q in range(n):
        c.rz(q, rng.uniform(0.0, TWO_PI))
    return c


def variational_ansatz(n: int, layers: int) -> Tuple[Circuit, np.ndarray]:
    """Circuit with placeholder angles 0 and the parameter index of every op
    (-1 for CX and barriers); parameters are ordered (layer, Ry for
    q=0..n-1, Rz for q=0..n-1).  A barrier closes each layer, which is what
    the adjoint's checkpointing counts layers by."""
    c = Circuit(n)
    pidx: List[int] = []
    k = 0
    for _ in range(layers):
        for q in range(n):
            c.ry(q, 0.0)
            pidx.append(k)
            k += 1
        for q in range(n):
            c.rz(q, 0.0)
            pidx.append(k)
            k += 1
        for q in range(n):
            c.cx(q, (q + 1) % n)
            pidx.append(-1)
        c.barrier()
        pidx.append(-1)
    return c, np.array(pidx, dtype=np.int32)


def random_pauli_sum(n: int, terms: int, seed: int = 11) -> List[Tuple[float, str]]:
    g = np.random.default_rng(seed)
    out = []
    for _ in range(terms):
        s = "".join("IXYZ"[i] for i in g.integers(0, 4, n))
        out.append((float(g.standard_normal()), s))
    return out


MIX = ["h", "s", "t", "rx", "ry", "rz", "u", "cx", "cz", "cp", "crz", "swap", "ccx", "cswap"]
_ARITY = {"h": 1, "s": 1, "t": 1, "rx": 1, "ry": 1, "rz": 1, "u": 1, "cx": 2, "cz": 2, "cp": 2,
          "crz": 2, "swap": 2, "ccx": 3, "cswap": 3}
_NPAR = {"rx": 1, "ry": 1, "rz": 1, "u": 3, "cp": 1, "crz": 1}


def random_mixed(n: int, depth: int, seed: int = 0) -> Circuit:
    """`depth` layers; each layer walks a random permutation of the qubits and
    places gates from the mix until every qubit has been used once."""
    g = np.random.default_rng(seed)
    c = Circuit(n)
    for _ in range(depth):
        perm = list(g.permutation(n))
        while perm:
            name = MIX[int(g.integers(0, len(MIX)))]
            a = _ARITY[name]
            if a > len(perm):
                continue
            qs = [int(perm.pop()) for _ in range(a)]
            ps = [float(x) for x in g.uniform(0.0, TWO_PI, _NPAR.get(name, 0))]
            getattr(c, name)(*qs, *ps)
    return c
