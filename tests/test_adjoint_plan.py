"""The tiled adjoint's plan, checked on the host.

ketgpu_adjoint_plan_describe returns the plan the tiled sweep kernels run:
blocks of gates, each with its tile qubits, its register phases and, per
gate, the encoded kind, register slots and control masks.  This test executes
that plan on the CPU with exactly the kernel's semantics: the thread/register
layout of each phase, the slot and mask encodings, and the per-thread
gradient sums. It checks the forward state and the gradients against the FP64
oracle, so a wrong encoding fails here, without a GPU.
"""
import math

import numpy as np
import pytest

from oracle.oracle import ARITY, CODE, GATES, NPARAMS, make_ops

TILE = {"c64": (12, 4), "c128": (11, 3)}
NTHREADS = 256


def _describe(n, ops, pidx, prec, ckpt=1):
    import ctypes as ct

    from ket_b200 import _lib
    lib = _lib.lib
    pid = np.ascontiguousarray(pidx, dtype=np.int32)
    length = ct.c_uint64()
    p = _lib.C64 if prec == "c64" else _lib.C128
    _lib.check(lib.ketgpu_adjoint_plan_describe(n, ops.ctypes.data, len(ops), pid.ctypes.data, p, ckpt, None, 0,
                                                ct.byref(length)))
    out = np.zeros(length.value, dtype=np.int32)
    _lib.check(lib.ketgpu_adjoint_plan_describe(n, ops.ctypes.data, len(ops), pid.ctypes.data, p, ckpt,
                                                out.ctypes.data, length.value, ct.byref(length)))
    v = list(out)
    k = 0
    blocks = []
    nb = v[k]
    k += 1
    for _ in range(nb):
        layer = v[k]
        pos = v[k + 1:k + 13]
        nph, ng = v[k + 13], v[k + 14]
        k += 15
        phases = []
        for _ in range(nph):
            phases.append((v[k:k + 4], v[k + 4], v[k + 5]))
            k += 6
        gates = []
        for _ in range(ng):
            f = v[k:k + 11]
            gates.append(dict(kind=f[0], s0=f[1], s1=f[2], tslot=f[3], tbit=f[4], cm_r=f[5], cm_g=f[6],
                              gen=f[7], real=f[8], grad=f[9], op=f[10]))
            k += 11
        blocks.append(dict(layer=layer, pos=pos, phases=phases, gates=gates))
    assert k == len(v)
    return blocks


def _deposit(x, positions):
    r = np.zeros_like(x)
    for b, p in enumerate(positions):
        r |= ((x >> b) & 1) << p
    return r


def _local_matrix(oracle, ops, i):
    """Full 2^k matrix of op i over its sorted qubits (oracle, FP64)."""
    qs = sorted(int(q) for q in ops[i]["q"][:ops[i]["nq"]])
    return oracle.block_matrix(ops[i:i + 1], qs), qs


def _gate_2x2(oracle, ops, i, g, tile_bits_of_ctrl, target_qubit, pos):
    M, qs = _local_matrix(oracle, ops, i)
    ctrl = 0
    for tb in tile_bits_of_ctrl:
        ctrl |= 1 << qs.index(pos[tb])
    tl = qs.index(target_qubit)
    if g["kind"] == 3:
        return M[ctrl, ctrl], M[ctrl | 1 << tl, ctrl | 1 << tl]
    m = np.array([[M[ctrl | a << tl, ctrl | b << tl] for b in (0, 1)] for a in (0, 1)])
    # the pair's amplitudes outside the controls subspace must be untouched
    return m


def _execute(oracle, n, ops, blocks, prec, psi, lam=None, reverse=False):
    """Run the plan's blocks (forward, or reverse with gradients) on host arrays."""
    TB, RB = TILE[prec]
    NR = 1 << RB
    grads = {}
    order = range(len(blocks) - 1, -1, -1) if reverse else range(len(blocks))
    for bi in order:
        b = blocks[bi]
        pos = b["pos"][:TB]
        rest = [q for q in range(n) if q not in pos]
        tiles = np.arange(1 << (n - TB), dtype=np.int64)
        base = _deposit(tiles, rest)
        e = np.arange(1 << TB, dtype=np.int64)
        idx = base[:, None] | _deposit(e, pos)[None, :]
        P = psi[idx]
        L = lam[idx] if reverse else None
        phases = list(enumerate(b["phases"]))
        if reverse:
            phases = phases[::-1]
        for _, (r, first, count) in phases:
            r = r[:RB]
            rmask = sum(1 << x for x in r)
            nonr = [t for t in range(TB) if not (rmask >> t) & 1]
            tid = np.arange(NTHREADS, dtype=np.int64)
            gbase = _deposit(tid, nonr)
            js = np.arange(NR, dtype=np.int64)
            E = gbase[:, None] | _deposit(js, r)[None, :]
            p = P[:, E]
            q = L[:, E] if reverse else None
            seq = range(first, first + count)
            if reverse:
                seq = reversed(seq)
            for gi in seq:
                g = b["gates"][gi]
                gok = (gbase & g["cm_g"]) == g["cm_g"]
                ctrl_tb = [t for t in range(TB) if (g["cm_g"] >> t) & 1] + \
                          [r[s] for s in range(RB) if (g["cm_r"] >> s) & 1]
                part = np.zeros(NTHREADS)
                if g["kind"] == 3:
                    tq = pos[g["tbit"]]
                    if g["tslot"] >= 0:
                        assert r[g["tslot"]] == g["tbit"]
                    m0, m3 = _gate_2x2(oracle, ops, g["op"], g, ctrl_tb, tq, pos)
                    if reverse:
                        m0, m3 = np.conj(m0), np.conj(m3)
                    for j in range(NR):
                        if (j & g["cm_r"]) != g["cm_r"]:
                            continue
                        bit = ((j >> g["tslot"]) & 1) * np.ones(NTHREADS, dtype=np.int64) if g["tslot"] >= 0 \
                            else (gbase >> g["tbit"]) & 1
                        on = gok
                        ph = np.where(bit == 1, m3, m0)
                        if reverse and g["gen"]:
                            im = (np.conj(q[:, :, j]) * p[:, :, j]).imag
                            w = np.where(bit == 1, -1.0, 1.0) if g["gen"] == 3 else (bit == 1).astype(float)
                            part += np.where(on, (w * im).sum(axis=0), 0.0)
                        p[:, on, j] *= ph[on]
                        if reverse:
                            q[:, on, j] *= ph[on]
                elif g["kind"] == 2:
                    a, c = g["s0"], g["s1"]
                    assert a < c
                    for j in range(NR):
                        if not (j >> a) & 1 or (j >> c) & 1 or (j & g["cm_r"]) != g["cm_r"]:
                            continue
                        j1 = j ^ (1 << a) ^ (1 << c)
                        for arr in ([p, q] if reverse else [p]):
                            t = arr[:, gok, j].copy()
                            arr[:, gok, j] = arr[:, gok, j1]
                            arr[:, gok, j1] = t
                else:
                    s = g["s0"]
                    tq = pos[r[s]]
                    m = None
                    if g["kind"] == 0:
                        m = _gate_2x2(oracle, ops, g["op"], g, ctrl_tb, tq, pos)
                        if g["real"]:
                            assert np.abs(m.imag).max() == 0.0
                        if reverse:
                            m = m.conj().T
                    for j in range(NR):
                        if (j >> s) & 1 or (j & g["cm_r"]) != g["cm_r"]:
                            continue
                        j1 = j | (1 << s)
                        if g["kind"] == 1:
                            for arr in ([p, q] if reverse else [p]):
                                t = arr[:, gok, j].copy()
                                arr[:, gok, j] = arr[:, gok, j1]
                                arr[:, gok, j1] = t
                            continue
                        if reverse and g["gen"]:
                            a0, a1, l0, l1 = p[:, :, j], p[:, :, j1], q[:, :, j], q[:, :, j1]
                            if g["gen"] == 1:
                                g0, g1 = a1, a0
                            elif g["gen"] == 2:
                                g0, g1 = -1j * a1, 1j * a0
                            else:
                                g0, g1 = a0, -a1
                            v = (np.conj(l0) * g0 + np.conj(l1) * g1).imag.sum(axis=0)
                            part += np.where(gok, v, 0.0)
                        for arr in ([p, q] if reverse else [p]):
                            x0, x1 = arr[:, gok, j].copy(), arr[:, gok, j1].copy()
                            arr[:, gok, j] = m[0, 0] * x0 + m[0, 1] * x1
                            arr[:, gok, j1] = m[1, 0] * x0 + m[1, 1] * x1
                if reverse and g["grad"] >= 0:
                    grads[g["op"]] = part.sum()
            P[:, E] = p
            if reverse:
                L[:, E] = q
        psi[idx] = P
        if reverse:
            lam[idx] = L
    return grads


def _random_circuit(n, count, seed, barriers=3):
    rng = np.random.default_rng(seed)
    gs, pidx = [], []
    k = 0
    pool = [g for g in GATES if g in ARITY and ARITY[g] >= 1]
    for i in range(count):
        if barriers and i % (count // barriers + 1) == count // barriers:
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


@pytest.mark.parametrize("ckpt", [1, 2, 0])
@pytest.mark.parametrize("prec,n,seed", [("c128", 11, 1), ("c128", 13, 2), ("c64", 12, 3), ("c64", 14, 4)])
def test_tiled_plan_reproduces_the_oracle(oracle, prec, n, seed, ckpt):
    """ckpt: the checkpoint interval in barrier-delimited layers; with more
    than one layer per segment, blocks may run across a segment's layers."""
    ops, pidx, npar = _random_circuit(n, 90, seed)
    blocks = _describe(n, ops, pidx, prec, ckpt)
    if ckpt == 1:  # one layer per block
        layer_of = np.cumsum([o["type"] == CODE["Barrier"] for o in ops])
        for b in blocks:
            assert {int(layer_of[g["op"]]) for g in b["gates"]} == {b["layer"]}
    if prec == "c64":
        # complex64 phases keep register slot 0 for the pack bit: no pair gate
        # targets it and no gate uses it as a control
        for b in blocks:
            for g in b["gates"]:
                assert g["cm_r"] & 1 == 0
                if g["kind"] in (0, 1):
                    assert g["s0"] >= 1
                if g["kind"] == 2:
                    assert g["s0"] >= 1 and g["s1"] >= 1
    # every unitary op is in exactly one block, once
    seen = [g["op"] for b in blocks for g in b["gates"]]
    assert sorted(seen) == [i for i in range(len(ops)) if ops[i]["type"] != CODE["Barrier"]]
    # forward
    psi = np.zeros(1 << n, dtype=np.complex128)
    psi[0] = 1
    _execute(oracle, n, ops, blocks, prec, psi)
    ref = oracle.run(n, ops, fuse=0)
    assert np.abs(psi - ref).max() < 1e-12
    # reverse: gradients of a Pauli sum against the FP64 oracle adjoint
    from ket_b200.workloads import random_pauli_sum
    ham = random_pauli_sum(n, 6, seed=seed + 10)
    lam = np.zeros_like(psi)
    for c, pstr in ham:
        lam += c * _pauli_apply(pstr, psi)
    grads = _execute(oracle, n, ops, blocks, prec, psi, lam, reverse=True)
    theta = np.array([ops[i]["p"][0] for i in range(len(ops)) if pidx[i] >= 0])
    _, g_ref = oracle.adjoint(n, ops, pidx, theta, ham)
    got = np.zeros(npar)
    for opi, v in grads.items():
        got[pidx[opi]] += -2.0 * v if ops[opi]["type"] == CODE["CP"] else v
    assert np.abs(got - g_ref).max() < 1e-10
    # psi is back at |0...0>
    assert abs(abs(psi[0]) - 1) < 1e-10


def _pauli_apply(pstr, psi):
    """P|psi> for a Pauli string (rightmost character = qubit 0)."""
    n = len(pstr)
    out = psi.copy()
    idx = np.arange(len(psi))
    for q in range(n):
        c = pstr[n - 1 - q]
        if c == "I":
            continue
        bit = (idx >> q) & 1
        if c == "X":
            out = out[idx ^ (1 << q)]
        elif c == "Y":
            out = out[idx ^ (1 << q)] * np.where(((idx >> q) & 1) == 1, 1j, -1j)
        elif c == "Z":
            out = out * np.where(bit == 1, -1, 1)
    return out


def test_ansatz_layer_needs_three_tiles_at_24_qubits():
    """The 24-qubit Ry/Rz + CX-ring layer: three blocks of 12 tile qubits."""
    from ket_b200.workloads import variational_ansatz
    circ, pidx = variational_ansatz(24, 2)
    blocks = _describe(24, circ.to_ops(), pidx, "c64")
    assert len(blocks) == 6
    assert all(len(b["phases"]) <= 4 for b in blocks)


def test_ansatz_blocks_span_layers_only_when_that_saves_passes():
    """20 qubits, 8 layers, checkpoints every 2 layers: blocks that run
    across the two layers of a segment need 20 passes instead of 24; at 24
    qubits they would save none, and the per-layer plan is kept."""
    from ket_b200.workloads import variational_ansatz
    circ, pidx = variational_ansatz(20, 8)
    assert len(_describe(20, circ.to_ops(), pidx, "c64", 1)) == 24
    assert len(_describe(20, circ.to_ops(), pidx, "c64", 2)) == 20
    circ, pidx = variational_ansatz(24, 8)
    b2 = _describe(24, circ.to_ops(), pidx, "c64", 2)
    assert len(b2) == 24 and max(len(b["phases"]) for b in b2) <= 4
