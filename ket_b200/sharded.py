"""A state vector sharded over several GPUs: global-qubit swaps.

A 2^n state over W = 2^G ranks, one process per GPU: physical index bits
0..L-1 (L = n - G) address a rank's local amplitudes, bits L..n-1 are the
rank id.  Every logical qubit sits at a physical position.  Gates run on the
local amplitudes only, so before a gate on a qubit whose position is global
the driver swaps that position with a local one.

Swapping global position L + b with local position l moves, on every rank r,
the half of the local amplitudes whose bit l differs from bit b of r to the
partner rank r ^ (1 << b), into the same slots there (an amplitude keeps all
its other bits, and the two halves are enumerated in the same order), so a
swap is one pairwise exchange of 2^(L-1) amplitudes per rank: send/recv over
NCCL on GPUs, over gloo in the CPU tests.  Between swaps the gates run as one
plan of the single-GPU backend on the L local qubits (fused blocks, tensor
cores), so a stretch of local gates costs what it costs on one GPU.

Which local position gives way: the one whose logical qubit is needed
furthest in the future (or never), among those the gate itself does not use.
The schedule is built on the host before anything runs; it depends only on
the circuit and n, G, so every rank builds the same one and the ranks take
the same collective steps in the same order.

Pauli expectations: a term's X and Y factors on global positions are first
swapped to local positions (the state is unchanged, only the map moves); a Z
factor on a global position is the sign of the rank's bit there; each rank
then takes the local term's expectation over its own amplitudes and the
ranks' values are summed.

Sampling is inverse-CDF sampling in physical index order, in two levels:
a draw's uniform u (a position in the cumulative probability, as ket's
measure takes it for a normalised state) picks the rank from the FP64
running sum of the ranks' probabilities, and u less the mass of the ranks
before it is drawn by the rank's own sampling tree; the physical index is
mapped back to the logical qubits and the draws are gathered on rank 0 in
their order.

Scope: unitary gates (ket's H..CSWAP), run from |0...0>, Pauli terms and sums
with at most L X/Y factors per term, sampling, the squared norm, and a
gather of the whole state for checking.  ``schedule`` and ``exchange_half`` are
device-independent and tested with gloo ranks on CPU.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

_UNITARY_MAX = 23  # ket::GateType::CSwap; H..CSwap are the unitary gates


def _arity(t: int) -> int:
    if t < 0 or t > _UNITARY_MAX:
        raise ValueError(f"gate type {t}: only unitary gates run on a sharded state")
    return 1 if t <= 11 else (2 if t <= 21 else 3)


@dataclass
class Swap:
    """Exchange global position `glob` (>= L) with local position `loc`."""
    glob: int
    loc: int


@dataclass
class Apply:
    """Gates to run on the local amplitudes (qubits are local positions)."""
    ops: np.ndarray


def schedule(n: int, global_bits: int, ops: np.ndarray,
             start: Optional[Sequence[int]] = None) -> Tuple[List[Union[Swap, Apply]], List[int]]:
    """The steps that run `ops` (ketgpu_op records, logical qubits) on a
    state whose logical qubit q sits at physical position start[q] (default:
    q), and the positions afterwards."""
    L = n - global_bits
    if L < 3:
        raise ValueError("a sharded state needs at least 3 local qubits")
    pos = list(start) if start is not None else list(range(n))
    if sorted(pos) != list(range(n)):
        raise ValueError("start must be a permutation of the qubits")
    at = [0] * n
    for q, p in enumerate(pos):
        at[p] = q
    ops = np.ascontiguousarray(ops)
    qubits = []
    for o in ops:
        a = _arity(int(o["type"]))
        qubits.append([int(o["q"][j]) for j in range(a)])
    # next use of each logical qubit after op i: scan backwards
    nxt = [dict() for _ in range(len(ops) + 1)]
    cur: dict = {}
    for i in range(len(ops) - 1, -1, -1):
        nxt[i + 1] = dict(cur)
        for q in qubits[i]:
            cur[q] = i
    steps: List[Union[Swap, Apply]] = []
    seg: List[np.ndarray] = []

    def flush():
        if seg:
            steps.append(Apply(np.concatenate(seg)))
            seg.clear()

    for i, o in enumerate(ops):
        qs = qubits[i]
        for q in qs:
            if pos[q] < L:
                continue
            future = nxt[i + 1]
            victim = max((p for p in range(L) if at[p] not in qs),
                         key=lambda p: (future.get(at[p], len(ops) + 1), -p))
            flush()
            g = pos[q]
            steps.append(Swap(g, victim))
            v = at[victim]
            pos[q], pos[v] = victim, g
            at[victim], at[g] = q, v
        r = o.copy()
        for j, q in enumerate(qs):
            r["q"][j] = pos[q]
        seg.append(np.array([r], dtype=ops.dtype))
    flush()
    return steps, pos


def half_view(x, loc: int, mine: int):
    """The amplitudes of x (real, shape (2^L, 2)) whose local bit `loc` is
    1 - mine, as a strided view; both sides of a swap enumerate their halves
    in the same order (the other bits ascending)."""
    dim = x.shape[0]
    return x.view(dim >> (loc + 1), 2, 1 << loc, 2)[:, 1 - mine]


def exchange_half(x, loc: int, bit: int, rank: int, group=None):
    """One swap's data movement on this rank: x is the rank's amplitudes as
    a real tensor of shape (2^L, 2) (any device); the half whose local bit
    `loc` differs from bit `bit` of the rank goes to rank ^ (1 << bit) and
    the partner's matching half lands in its place."""
    import torch.distributed as dist
    partner = rank ^ (1 << bit)
    half = half_view(x, loc, (rank >> bit) & 1)
    send = half.contiguous()
    recv = send.new_empty(send.shape)
    reqs = dist.batch_isend_irecv([dist.P2POp(dist.isend, send, partner, group),
                                   dist.P2POp(dist.irecv, recv, partner, group)])
    for r in reqs:
        r.wait()
    half.copy_(recv)


class DeviceShard:
    """This rank's local amplitudes on its GPU (the single-GPU backend)."""

    def __init__(self, local_qubits: int, precision: str = "c64"):
        from .api import DeviceState
        self.state = DeviceState(local_qubits, precision)
        self.precision = precision

    def _stream(self):
        import torch
        from ._lib import lib
        return torch.cuda.ExternalStream(lib.ketgpu_state_stream(self.state.handle))

    def reset(self, holds_ground: bool):
        import torch
        if holds_ground:
            self.state.reset()
        else:
            with torch.cuda.stream(self._stream()):
                self.state.torch_view().zero_()

    def apply(self, ops: np.ndarray, options=None):
        self.state.apply(ops, options)

    def exchange(self, loc: int, bit: int, rank: int, group=None):
        import torch
        with torch.cuda.stream(self._stream()):
            exchange_half(torch.view_as_real(self.state.torch_view()), loc, bit, rank, group)

    def norm(self) -> float:
        return self.state.norm()

    def expval(self, pauli: str) -> float:
        """<psi|P|psi> over this rank's amplitudes (no normalisation)."""
        return self.state.expval(pauli)

    def sample(self, positions: np.ndarray) -> np.ndarray:
        """Local indices drawn by the state's sampling tree for positions in
        this rank's cumulative probability (absolute, like a uniform for a
        normalised state)."""
        return self.state.sample(positions)

    def to_numpy(self) -> np.ndarray:
        return self.state.to_numpy()

    def close(self):
        self.state.close()


class ShardedState:
    """A 2^n state over the ranks of `group` (a power of two of them), each
    holding 2^(n - G) amplitudes in `shard` (default: on its GPU)."""

    def __init__(self, n_qubits: int, precision: str = "c64", group=None, shard=None):
        import torch.distributed as dist
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        if self.world & (self.world - 1):
            raise ValueError("the number of ranks must be a power of two")
        self.n = int(n_qubits)
        self.global_bits = self.world.bit_length() - 1
        self.local_qubits = self.n - self.global_bits
        self.shard = shard if shard is not None else DeviceShard(self.local_qubits, precision)
        self.pos = list(range(self.n))
        self.swaps = 0
        self.reset()

    def reset(self):
        """|0...0>: the amplitude 1 sits on rank 0 at local index 0."""
        self.shard.reset(self.rank == 0)
        self.pos = list(range(self.n))

    def apply(self, circuit, options=None) -> "ShardedState":
        from .circuit import Circuit
        ops = circuit.to_ops() if isinstance(circuit, Circuit) else np.ascontiguousarray(circuit)
        steps, pos = schedule(self.n, self.global_bits, ops, self.pos)
        L = self.local_qubits
        for st in steps:
            if isinstance(st, Swap):
                self.shard.exchange(st.loc, st.glob - L, self.rank, self.group)
                self.swaps += 1
            else:
                self.shard.apply(st.ops, options)
        self.pos = pos
        return self

    def run(self, circuit, options=None) -> "ShardedState":
        self.reset()
        return self.apply(circuit, options)

    def _sum_over_ranks(self, x: float) -> float:
        import torch
        import torch.distributed as dist
        v = torch.tensor([float(x)], dtype=torch.float64)
        if self.world > 1:
            if dist.get_backend(self.group) == "nccl":
                v = v.cuda()
            dist.all_reduce(v, group=self.group)
        return float(v.item())

    def norm(self) -> float:
        """Squared norm of the whole state (sum over ranks)."""
        return self._sum_over_ranks(self.shard.norm())

    def expval(self, obs) -> float:
        """<psi|P|psi> for a Pauli string (n characters of I X Y Z, the
        rightmost for qubit 0, as ket writes them) or a sum of
        (coefficient, string) terms."""
        terms = [(1.0, obs)] if isinstance(obs, str) else [(float(c), str(p)) for c, p in obs]
        return sum(c * self._expval_term(p) for c, p in terms)

    def sample(self, uniforms) -> Optional[np.ndarray]:
        """Basis-state indices (logical qubit order) drawn for the uniforms in
        [0, 1), the same on every rank, as ket's measure draws them from a
        normalised state; on rank 0 (None elsewhere)."""
        import torch.distributed as dist
        u = np.ascontiguousarray(uniforms, dtype=np.float64)
        mine_p = float(self.shard.norm())
        if self.world > 1:
            tot = [None] * self.world
            dist.all_gather_object(tot, mine_p, group=self.group)
        else:
            tot = [mine_p]
        tot = np.array(tot, dtype=np.float64)
        cum = np.cumsum(tot)
        if not cum[-1] > 0:
            raise ValueError("cannot sample a state of zero norm")
        x = u
        # the first rank whose running sum exceeds x (ranks without
        # probability never qualify); x at the very top goes to the last
        # rank with probability
        last = int(np.nonzero(tot > 0)[0].max())
        which = np.minimum(np.searchsorted(cum, x, side="right"), last)
        sel = np.nonzero(which == self.rank)[0]
        local = np.empty(0, dtype=np.uint64)
        if len(sel):
            lo = cum[self.rank] - tot[self.rank]
            local = np.asarray(self.shard.sample(np.maximum(x[sel] - lo, 0.0)), dtype=np.uint64)
        phys = (np.uint64(self.rank) << np.uint64(self.local_qubits)) | local
        logical = np.zeros_like(phys)
        for q, p in enumerate(self.pos):
            logical |= ((phys >> np.uint64(p)) & np.uint64(1)) << np.uint64(q)
        if self.world > 1:
            parts = [None] * self.world if self.rank == 0 else None
            dist.gather_object((sel, logical), parts, dst=0, group=self.group)
        else:
            parts = [(sel, logical)]
        if self.rank != 0:
            return None
        out = np.empty(len(u), dtype=np.uint64)
        for sl, lg in parts:
            out[sl] = lg
        return out

    def _expval_term(self, pauli: str) -> float:
        n, L = self.n, self.local_qubits
        if len(pauli) != n:
            raise ValueError(f"Pauli string of length {len(pauli)} for {n} qubits")
        ch = [pauli[n - 1 - q].upper() for q in range(n)]
        if any(c not in "IXYZ" for c in ch):
            raise ValueError("Pauli strings hold only I, X, Y and Z")
        if sum(c in "XY" for c in ch) > L:
            raise ValueError("a sharded state takes at most n - G X/Y factors per term")
        at = [0] * n
        for q, p in enumerate(self.pos):
            at[p] = q
        # X and Y factors must act on local positions: swap them in, giving
        # way with local positions whose factor is I (else Z)
        for q in range(n):
            if ch[q] not in "XY" or self.pos[q] < L:
                continue
            victim = min((p for p in range(L) if ch[at[p]] not in "XY"), key=lambda p: (ch[at[p]] != "I", p))
            g = self.pos[q]
            self.shard.exchange(victim, g - L, self.rank, self.group)
            self.swaps += 1
            v = at[victim]
            self.pos[q], self.pos[v] = victim, g
            at[victim], at[g] = q, v
        sign = 1.0
        for q in range(n):
            if ch[q] == "Z" and self.pos[q] >= L and (self.rank >> (self.pos[q] - L)) & 1:
                sign = -sign
        local = "".join(ch[at[p]] for p in range(L - 1, -1, -1))
        return self._sum_over_ranks(sign * self.shard.expval(local))

    def gather(self) -> Optional[np.ndarray]:
        """The whole state in logical qubit order, on rank 0 (None elsewhere)."""
        import torch.distributed as dist
        local = self.shard.to_numpy()
        parts = [None] * self.world if self.rank == 0 else None
        if self.world > 1:
            dist.gather_object(local, parts, dst=0, group=self.group)
        else:
            parts = [local]
        if self.rank != 0:
            return None
        phys = np.concatenate(parts)  # physical index = rank << L | local
        n = self.n
        # numpy axis k of the (2,)*n view is index bit n-1-k; logical bit q
        # is physical bit pos[q]
        t = phys.reshape((2,) * n)
        axes = [n - 1 - self.pos[n - 1 - k] for k in range(n)]
        return np.ascontiguousarray(t.transpose(axes)).reshape(-1)

    def close(self):
        self.shard.close()
