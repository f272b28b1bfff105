"""The sharded state (ket_b200/sharded.py) on CPU: the swap schedule and the
qubit map, emulated in one process, and the real exchange between gloo ranks
(world size 2 and 4).  Each rank's local gates run on the oracle, so these
tests check the host logic and the data movement, not the GPU kernels; the
results are compared with the oracle's unsharded state."""
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _circuits(n):
    from ket_b200.workloads import random_brickwork, random_mixed
    return [random_brickwork(n, 6, seed=3).to_ops(), random_mixed(n, 8, seed=11).to_ops()]


def _emulate(n, G, ops, oracle):
    """Run the schedule on all 2^G ranks' slices of one array (physical
    order) and return the state in logical order."""
    from ket_b200 import sharded
    L = n - G
    steps, pos = sharded.schedule(n, G, ops)
    phys = np.zeros(1 << n, dtype=np.complex128)
    phys[0] = 1.0
    swaps = 0
    for st in steps:
        if isinstance(st, sharded.Apply):
            for r in range(1 << G):
                sl = slice(r << L, (r + 1) << L)
                phys[sl] = oracle.apply(L, phys[sl], st.ops, fuse=0)
        else:  # swap physical bits st.glob and st.loc
            idx = np.arange(1 << n)
            bg, bl = (idx >> st.glob) & 1, (idx >> st.loc) & 1
            src = idx ^ ((bg ^ bl) << st.glob) ^ ((bg ^ bl) << st.loc)
            phys = phys[src]
            swaps += 1
    t = phys.reshape((2,) * n)
    return np.ascontiguousarray(t.transpose([n - 1 - pos[n - 1 - k] for k in range(n)])).reshape(-1), swaps


@pytest.mark.parametrize("G", [1, 2, 3])
def test_schedule_emulated_matches_unsharded(oracle, G):
    n = 11
    for ops in _circuits(n):
        got, swaps = _emulate(n, G, ops, oracle)
        want = oracle.run(n, ops, fuse=0)
        assert np.abs(got - want).max() < 1e-12
        assert swaps > 0


def test_schedule_local_gates_need_no_swap():
    from ket_b200 import sharded
    from ket_b200.circuit import Circuit
    c = Circuit(8)
    for q in range(6):
        c.h(q)
    c.cx(0, 5)
    steps, pos = sharded.schedule(8, 2, c.to_ops())
    assert len(steps) == 1 and isinstance(steps[0], sharded.Apply) and pos == list(range(8))
    c.h(7)  # a global qubit: one swap, with the local position used furthest ahead (never: any)
    steps, pos = sharded.schedule(8, 2, c.to_ops())
    swaps = [s for s in steps if isinstance(s, sharded.Swap)]
    assert len(swaps) == 1 and swaps[0].glob == 7 and pos[7] < 6
    with pytest.raises(ValueError):
        sharded.schedule(4, 2, c.to_ops())  # fewer than 3 local qubits
    m = Circuit(8)
    m.measure(0, 0)
    with pytest.raises(ValueError):
        sharded.schedule(8, 1, m.to_ops())


class OracleShard:
    """A rank's local amplitudes in host memory, gates on the oracle."""

    def __init__(self, L):
        import sys
        sys.path.insert(0, ROOT)
        from oracle.oracle import Oracle
        self.L = L
        self.a = np.zeros(1 << L, dtype=np.complex128)
        self.oracle = Oracle()

    def reset(self, holds_ground):
        self.a[:] = 0
        if holds_ground:
            self.a[0] = 1.0

    def apply(self, ops, options=None):
        self.a[:] = self.oracle.apply(self.L, self.a, ops, fuse=0)

    def exchange(self, loc, bit, rank, group=None):
        import torch
        from ket_b200.sharded import exchange_half
        exchange_half(torch.from_numpy(self.a.view(np.float64).reshape(-1, 2)), loc, bit, rank, group)

    def norm(self):
        return float(np.vdot(self.a, self.a).real)

    def expval(self, pauli):
        return self.oracle.expval(self.L, self.a, pauli)

    def sample(self, u):
        return self.oracle.sample_tree(self.L, self.a, u)

    def to_numpy(self):
        return self.a.copy()

    def close(self):
        pass


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


# n = 10: X/Y/Z on the top (global) qubits, on low ones, and mixed
_PAULIS = ["XIIIIIIIIZ", "YZIIIIIIIX", "ZZIIIIIIII", "IIIIXYZIII", "XYZXYZIIII", "ZIIIIIIIIY", "IIIIIIIIII"]
_COEFFS = [0.5, -1.25, 2.0, 0.75, -0.3, 1.1, 0.2]


def _worker(rank, world, port, n, q):
    import datetime
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    from ket_b200.sharded import ShardedState
    out = []
    for ops in _circuits(n):
        G = world.bit_length() - 1
        s = ShardedState(n, shard=OracleShard(n - G))
        s.run(ops)
        ev = [s.expval(p) for p in _PAULIS] + [s.expval(list(zip(_COEFFS, _PAULIS)))]
        draws = s.sample(np.random.default_rng(17).random(20000))
        out.append((s.gather(), s.norm(), s.swaps, ev, draws, list(s.pos)))
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, out))


@pytest.mark.parametrize("world", [2, 4])
def test_sharded_run_on_gloo_ranks(oracle, world):
    import torch.multiprocessing as mp
    n = 10
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, n, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=300) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for i, ops in enumerate(_circuits(n)):
        want = oracle.run(n, ops, fuse=0)
        got, norm, swaps, ev, _, pos = res[0][i]
        assert np.abs(got - want).max() < 1e-12
        assert swaps > 0
        exp = [oracle.expval(n, want, p) for p in _PAULIS]
        exp.append(sum(c * e for c, e in zip(_COEFFS, exp)))
        for r in range(world):
            assert np.allclose(res[r][i][3], exp, atol=1e-12), (r, res[r][i][3], exp)
            if r:
                assert res[r][i][4] is None
        # draws: valid outcomes, distributed as |psi|^2 -- counts within 6
        # sigma plus 3 (outcomes with a fraction of an expected draw are in
        # the Poisson regime, where one draw is not an outlier)
        draws = res[0][i][4]
        p = np.abs(want) ** 2
        N = len(draws)
        assert N == 20000 and np.all(p[draws.astype(np.int64)] > 0)
        counts = np.bincount(draws.astype(np.int64), minlength=1 << n)
        assert np.all(np.abs(counts - N * p) <= 6 * np.sqrt(N * p * (1 - p)) + 3)
        # and they are the inverse CDF of the state in physical index order
        # (the ranks' trees sum in another order than numpy, so a draw on a
        # boundary may differ by rounding)
        idx = np.arange(1 << n)
        lidx = np.zeros_like(idx)
        for qq, pp in enumerate(pos):
            lidx |= ((idx >> pp) & 1) << qq
        cdf = np.cumsum(np.abs(got[lidx]) ** 2)
        u = np.random.default_rng(17).random(N)
        ref = lidx[np.minimum(np.searchsorted(cdf, u, side="right"), (1 << n) - 1)]
        assert np.sum(ref != draws.astype(np.int64)) <= 5
        for r in range(world):
            assert abs(res[r][i][1] - 1.0) < 1e-12  # every rank sees the all-reduced norm
            assert res[r][i][2] == swaps             # and took the same steps
            if r:
                assert res[r][i][0] is None


@pytest.mark.gpu
def test_device_shards_emulate_two_ranks_on_one_gpu(oracle):
    """The device side of a 2-rank run on one GPU: two DeviceShards (the
    single-GPU kernels on 2^(n-1) amplitudes each) follow the schedule, and a
    swap exchanges their halves in place through the same strided views the
    NCCL exchange sends from and receives into."""
    import torch
    import ket_b200 as ket
    from ket_b200 import sharded
    from ket_b200.workloads import random_brickwork
    n, G = 14, 1
    L = n - G
    ops = random_brickwork(n, 8, seed=5).to_ops()
    steps, pos = sharded.schedule(n, G, ops)
    shards = [sharded.DeviceShard(L, "c128"), sharded.DeviceShard(L, "c128")]
    shards[0].reset(True)
    shards[1].reset(False)
    opt = ket.make_options("c128", "greedy", 5, True)
    swaps = 0
    for st in steps:
        if isinstance(st, sharded.Apply):
            for sh in shards:
                sh.apply(st.ops, opt)
        else:
            assert st.glob == L
            torch.cuda.synchronize()
            h0 = sharded.half_view(torch.view_as_real(shards[0].state.torch_view()), st.loc, 0)
            h1 = sharded.half_view(torch.view_as_real(shards[1].state.torch_view()), st.loc, 1)
            tmp = h0.clone()
            h0.copy_(h1)
            h1.copy_(tmp)
            torch.cuda.synchronize()
            swaps += 1
    assert swaps > 0
    phys = np.concatenate([shards[0].to_numpy(), shards[1].to_numpy()])
    got = np.ascontiguousarray(phys.reshape((2,) * n).transpose([n - 1 - pos[n - 1 - k] for k in range(n)])).reshape(-1)
    want = oracle.run(n, ops, fuse=0)
    assert np.abs(got - want).max() < 1e-12
    assert abs(sum(sh.norm() for sh in shards) - 1.0) < 1e-12
    for sh in shards:
        sh.close()


@pytest.mark.gpu
def test_sharded_state_on_one_rank_is_the_device_state(oracle):
    """World size 1: no global qubits, no swaps; the state is the device
    backend's, in complex64 on the tensor cores."""
    import ket_b200 as ket
    from ket_b200.sharded import ShardedState
    from ket_b200.workloads import random_brickwork
    n = 16
    ops = random_brickwork(n, 8, seed=2).to_ops()
    s = ShardedState(n, "c64")
    s.run(ops, ket.make_options("c64", "greedy", 6, True))
    got = s.gather()
    assert s.swaps == 0 and abs(s.norm() - 1.0) < 1e-6
    want = oracle.run(n, ops, fuse=0)
    assert np.abs(got - want).max() < 1e-5
    s.close()


def test_schedule_with_three_local_qubits(oracle):
    """The fewest local qubits a sharded state allows (3): a 3-qubit gate on
    global qubits swaps every local position out."""
    from ket_b200 import sharded
    from ket_b200.circuit import Circuit
    from ket_b200.workloads import random_mixed
    n, G = 6, 3
    c = Circuit(n)
    c.h(3)
    c.h(4)
    c.h(5)
    c.ccx(3, 4, 5)
    c.cswap(5, 0, 4)
    ops = np.concatenate([c.to_ops(), random_mixed(n, 6, seed=9).to_ops()])
    steps, pos = sharded.schedule(n, G, ops)
    got, swaps = _emulate(n, G, ops, oracle)
    assert np.abs(got - oracle.run(n, ops, fuse=0)).max() < 1e-12
    assert swaps >= 3


def test_schedule_property_over_random_circuits(oracle):
    """Property check of the swap schedule: for random circuits, register
    sizes and numbers of global qubits, running the steps on the ranks'
    slices reproduces the unsharded state, and running the same circuit again
    from the map the first run left (a second apply) still does."""
    from ket_b200 import sharded
    from ket_b200.workloads import random_mixed
    rng = np.random.default_rng(2024)
    for trial in range(24):
        n = int(rng.integers(6, 12))
        G = int(rng.integers(1, min(4, n - 3) + 1))
        ops = random_mixed(n, int(rng.integers(2, 10)), seed=int(rng.integers(1 << 30))).to_ops()
        got, _ = _emulate(n, G, ops, oracle)
        assert np.abs(got - oracle.run(n, ops, fuse=0)).max() < 1e-12, (trial, n, G)
        # a second application starting from the first run's map
        steps1, pos1 = sharded.schedule(n, G, ops)
        steps2, pos2 = sharded.schedule(n, G, ops, start=pos1)
        assert sorted(pos2) == list(range(n))
        for st in steps2:
            if isinstance(st, sharded.Apply):
                for o in st.ops:
                    a = 1 if o["type"] <= 11 else (2 if o["type"] <= 21 else 3)
                    assert all(int(o["q"][j]) < n - G for j in range(a))
