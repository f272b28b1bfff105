"""Host-side checks that need no GPU: the C ABI library loads and exports
every symbol of include/ket_b200.h, the circuit recorder mirrors ket's
validation, the uniform streams agree, and the planner (host code) builds
the expected plans."""
import ctypes as ct
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "ket_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ketgpu_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from ket_b200 import _lib
    names = header_functions()
    assert len(names) >= 30
    for name in names:
        assert hasattr(_lib.lib, name), name
    assert _lib.lib.ketgpu_abi_version() == 1


def test_circuit_validation_mirrors_ket():
    import ket_b200 as ket
    c = ket.Circuit(3)
    with pytest.raises(IndexError):
        c.x(3)
    with pytest.raises(ValueError):
        c.ccx(0, 1, 0)
    with pytest.raises(ValueError):
        c.append(ket.Circuit(2), [0])
    c.measure(2, 5)
    assert c.n_clbits == 6
    c.probe()
    c.probe("x")
    assert [g.label for g in c.gates if g.type == ket.GateType.Probe] == ["ψ0", "x"]


def test_op_layout_and_codes():
    import ket_b200 as ket
    from ket_b200._lib import OP_DTYPE
    assert OP_DTYPE.itemsize == 48
    c = ket.Circuit(3)
    c.cu(2, 0, 0.1, 0.2, 0.3)
    c.measure(1, 4)
    ops = c.to_ops()
    assert ops[0]["type"] == 19 and list(ops[0]["q"][:2]) == [2, 0]
    assert list(ops[0]["p"]) == [0.1, 0.2, 0.3]
    assert ops[1]["type"] == 24 and ops[1]["q"][1] == 4


def test_clifford_detection():
    import ket_b200 as ket
    c = ket.Circuit(2)
    for g in ("h", "x", "y", "z", "s", "sdg"):
        getattr(c, g)(0)
    c.cx(0, 1)
    c.cy(1, 0)
    c.cz(0, 1)
    c.swap(0, 1)
    c.barrier()
    c.measure_all()
    assert ket.is_clifford(c) and ket.chosen_method(c) == "stabilizer"
    sub = ket.Circuit(1)
    sub.t(0)
    c.append(sub, [1])
    assert not ket.is_clifford(c)


def test_uniform_streams_agree(oracle):
    import ket_b200 as ket
    from ket_b200.workloads import MT19937
    for seed in (0, 1, 42, 2**32 - 1):
        a = ket.uniforms(seed, 1500)
        assert np.array_equal(a, oracle.uniforms(seed, 1500))
        r = MT19937(seed)
        assert [r.canonical() for _ in range(3)] == list(a[:3])


def test_plans_on_the_host():
    import ket_b200 as ket
    from ket_b200.workloads import random_brickwork
    c = random_brickwork(30, 40)
    un = ket.plan_stats(c, ket.make_options("c64", "none"))
    gr = ket.plan_stats(c, ket.make_options("c64", "greedy", 5, True))
    # the plain method: one pass per gate, except that per layer the U gates
    # on qubits 0..10 and the CX gates within qubits 0..10 each share one
    # shared-memory pass (1780 gates, 1780 - 40 * (11 - 1) - 40 * (5 - 1) passes)
    assert un["n_gates"] == 1780 and un["n_passes"] == 1220
    assert gr["n_passes"] < un["n_passes"] / 7
    assert gr["n_tensor"] == gr["n_fused"] > 0
    # algorithmic bytes: 760 dense 1q passes + 380 CX passes over half the
    # state + 80 shared-memory runs over the whole state
    assert un["bytes"] == 760 * 16 * 2**30 + 380 * 8 * 2**30 + 80 * 16 * 2**30
    assert gr["bytes"] < un["bytes"] / 6


def test_pass_qubits_describe_the_blocks():
    """Each dense block of the 30-qubit brick wall reports its qubits in
    ascending order; together the blocks cover every qubit."""
    import ket_b200 as ket
    from ket_b200.api import Plan
    from ket_b200.workloads import random_brickwork
    c = random_brickwork(30, 40)
    p = Plan(30, c.to_ops(), ket.make_options("c64", "greedy", 5, True))
    seen = set()
    n_tc = 0
    for i in range(p.stats()["n_passes"]):
        info, qs = p.pass_info(i), p.pass_qubits(i)
        if info["kind"] == 2:
            assert len(qs) == info["k"] and qs == sorted(set(qs)) and 0 <= qs[0] and qs[-1] < 30
            n_tc += info["tensor"]
            seen |= set(qs)
        elif info["kind"] in (3, 4):
            assert qs == []
        else:
            assert 1 <= len(qs) <= 3
    assert n_tc == 114 and seen == set(range(30))
    with pytest.raises(Exception):
        p.pass_qubits(10**6)


def test_tensor_core_producer_forms():
    """Which tensor-core blocks fetch tiles with one tensor copy (and how many
    tensor-map dimensions), and which store straight from registers: the
    first tensor-copy dimension is qubits 0-3, later ones hold runs of at
    most 8 tile qubits, at most 5 in all; blocks targeting qubit 0 keep the
    cp.async producers, and blocks whose lowest target is qubit 1 take the
    tensor copy only when their converter reads stay conflict-free (1 3 5 7 9
    and 1 2 25 26 27 do, measured 4.6 -> 5.8-5.9 TB/s; 1 2 3 4 5 does not,
    measured 4.9 -> 4.4 TB/s)."""
    import collections
    import ket_b200 as ket
    from ket_b200.api import Plan
    from ket_b200.workloads import random_brickwork
    opt = ket.make_options("c64", "greedy", 5, True)
    p = Plan(30, random_brickwork(30, 40).to_ops(), opt)
    forms = collections.Counter()
    for i in range(p.stats()["n_passes"]):
        info = p.pass_info(i)
        if info["kind"] == 2 and info["tensor"]:
            f = p.pass_tc_form(i)
            forms[(f["tma_dims"], f["direct"])] += 1
            if f["tma_dims"]:
                assert p.pass_qubits(i)[0] >= 1 and f["direct"]
        else:
            with pytest.raises(ValueError):
                p.pass_tc_form(i)
    assert forms == {(2, True): 21, (3, True): 68, (4, True): 9, (0, False): 16}
    # 4-qubit blocks (11-qubit tiles): the same rule
    p4 = Plan(30, random_brickwork(30, 40).to_ops(), ket.make_options("c64", "greedy", 4, True))
    for i in range(p4.stats()["n_passes"]):
        info = p4.pass_info(i)
        if info["kind"] == 2 and info["tensor"]:
            assert info["k"] == 4
            f = p4.pass_tc_form(i)
            assert 0 <= f["tma_dims"] <= 5
            low = p4.pass_qubits(i)[0]
            assert (f["tma_dims"] > 0) == (low >= 2) or low == 1
            assert f["direct"] or f["tma_dims"] == 0

    expect = {(10, 11, 12, 13, 14): (3, True), (5, 6, 23, 24, 25): (3, True), (8, 9, 10, 13, 14): (4, True),
              (2, 3, 4, 5, 6): (2, True), (3, 4, 5, 14, 15): (3, True), (8, 10, 12, 14, 16): (0, True),
              (3, 9, 14, 20, 27): (0, True), (1, 3, 5, 7, 9): (2, True), (1, 2, 25, 26, 27): (3, True),
              (1, 2, 3, 4, 5): (0, False), (0, 1, 2, 3, 4): (0, False)}
    for qs, want in expect.items():
        c = ket.Circuit(28)
        for q in qs:
            c.u(q, 0.3, 0.2, 0.1)
        for a, b in zip(qs[:-1], qs[1:]):
            c.cx(a, b)
        p = Plan(28, c.to_ops(), opt)
        tc = [i for i in range(p.stats()["n_passes"]) if p.pass_info(i)["tensor"]]
        assert len(tc) == 1 and tuple(p.pass_qubits(tc[0])) == qs
        f = p.pass_tc_form(tc[0])
        assert (f["tma_dims"], f["direct"]) == want, qs


def test_thread_count_api_like_ket():
    """set_num_threads / num_threads behave as ket's (src/parallelism.cpp:164-169,
    tests/test_parallelism.cpp:102-109): the default is 1, 0 means every
    hardware thread, and the value reads back."""
    import subprocess
    import sys
    import ket_b200 as ket
    fresh = subprocess.run([sys.executable, "-c", "import ket_b200 as k; print(k.num_threads())"],
                           capture_output=True, text=True, check=True)
    assert fresh.stdout.strip() == "1"
    try:
        ket.set_num_threads(4)
        assert ket.num_threads() == 4
        ket.set_num_threads(0)
        assert ket.num_threads() >= 1
        ket.set_num_threads(1)
        assert ket.num_threads() == 1
    finally:
        ket.set_num_threads(1)


def test_release_cache_without_a_kept_state():
    """ketgpu_release_cache is a no-op (and touches no device) when no
    ketgpu_run call has kept a state."""
    from ket_b200 import _lib
    assert _lib.lib.ketgpu_release_cache() == 0
    assert _lib.lib.ketgpu_release_cache() == 0


def test_diagonal_runs_in_the_plan():
    """The 33-qubit QFT-pattern circuit: the 528 CP gates form one diagonal
    pass; the brick wall (no diagonal gates) is planned as before."""
    import ctypes as ct

    import ket_b200 as ket
    from ket_b200 import _lib
    from ket_b200.workloads import qft_ghz_rz
    c = qft_ghz_rz(33)
    opt = ket.make_options("c64", "greedy", 5, True)
    st = ket.plan_stats(c, opt)
    assert st["n_passes"] <= 20 and st["n_gates"] == 627
    ops = c.to_ops()
    h = ct.c_void_p()
    _lib.check(_lib.lib.ketgpu_plan_create(33, ops.ctypes.data, len(ops), ct.byref(opt), ct.byref(h)))
    kinds = []
    for i in range(st["n_passes"]):
        kind, k, tc, b = ct.c_int32(), ct.c_int32(), ct.c_int32(), ct.c_double()
        _lib.check(_lib.lib.ketgpu_plan_pass_info(h, i, ct.byref(kind), ct.byref(k), ct.byref(tc), ct.byref(b)))
        kinds.append((kind.value, k.value))
    _lib.lib.ketgpu_plan_destroy(h)
    diag = [k for kind, k in kinds if kind == 4]
    assert diag == [33]
    # no diagonal runs without fusion, or with ket's own Fuser rule
    for mode in ("none", "reference"):
        assert ket.plan_stats(c, ket.make_options("c64", mode))["n_passes"] > 400


def test_plan_errors():
    import ket_b200 as ket
    from ket_b200 import _lib
    ops = np.zeros(1, dtype=_lib.OP_DTYPE)
    ops[0]["type"] = 13
    ops[0]["q"][:2] = [0, 5]
    h = ct.c_void_p()
    opt = ket.make_options("c64")
    rc = _lib.lib.ketgpu_plan_create(3, ops.ctypes.data, 1, ct.byref(opt), ct.byref(h))
    assert rc == _lib.ERR_OUT_OF_RANGE
    assert "out of range" in _lib.lib.ketgpu_last_error().decode()
    ops[0]["q"][:2] = [1, 1]
    rc = _lib.lib.ketgpu_plan_create(3, ops.ctypes.data, 1, ct.byref(opt), ct.byref(h))
    assert rc == _lib.ERR_INVALID
    bad = ket.make_options("c64", "greedy", 9)
    ops[0]["q"][:2] = [0, 1]
    assert _lib.lib.ketgpu_plan_create(3, ops.ctypes.data, 1, ct.byref(bad), ct.byref(h)) == _lib.ERR_INVALID


def test_workload_shapes():
    from ket_b200.workloads import qft_ghz_rz, random_mixed, variational_ansatz
    c = qft_ghz_rz(33)
    assert len(c.gates) == 33 + 528 + 1 + 32 + 33
    a, pidx = variational_ansatz(24, 8)
    assert (pidx >= 0).sum() == 384 and len(a.gates) == 8 * 73
    m = random_mixed(22, 20, seed=3)
    used = sum(len(g.qubits) for g in m.gates)
    assert used == 22 * 20


def test_cost_model_features_on_the_host():
    import ctypes as ct
    from ket_b200 import _lib
    import ket_b200 as ket
    c = ket.Circuit(20)
    c.h(0)
    c.cx(0, 5)
    c.cp(5, 19, 0.3)
    ops = c.to_ops()
    f = np.zeros(48, dtype=np.float32)
    _lib.check(_lib.lib.ketgpu_block_features(20, _lib.C64, ops.ctypes.data, len(ops), 1, 1, f.ctypes.data))
    assert f[2] == 1 and f[3] == 1 and abs(f[4] - 3 / 6) < 1e-6 and f[47] == 1
    assert f[34] == 1 and f[39] == 1 and f[42] == 1        # qubit 0, qubit 5, top qubit
    assert abs(f[20] + f[6 + 20] + f[8 + 20] - 3 / 16) < 1e-6  # H, CX, CP counted
    g = np.zeros(48, dtype=np.float32)
    _lib.check(_lib.lib.ketgpu_block_features(20, _lib.C64, ops[2:].ctypes.data, 1, 0, 0, g.ctypes.data))
    assert g[2] == 0 and abs(g[12] - 0.25) < 1e-6           # CP alone: a quarter of the state
    assert _lib.lib.ketgpu_block_features(20, _lib.C64, ops.ctypes.data, 3, 0, 0, g.ctypes.data) == _lib.ERR_INVALID


def test_learned_mode_without_a_model_falls_back_to_greedy():
    import ket_b200 as ket
    from ket_b200.workloads import random_mixed
    c = random_mixed(24, 12, seed=4)
    a = ket.plan_stats(c, ket.make_options("c64", "greedy", 5, True))
    b = ket.plan_stats(c, ket.make_options("c64", "learned", 5, True))
    assert a["n_passes"] == b["n_passes"] and a["bytes"] == b["bytes"]


def test_reference_harness_builds_the_bench_circuit(reference, oracle):
    """The reference arm of the benchmark generates the 30-qubit brick wall
    without the B200 package; it must be the circuit the B200 arm times."""
    from oracle.oracle import brickwork_ops
    from ket_b200.workloads import random_brickwork
    for n, depth, seed in ((30, 40, 1234), (7, 5, 3)):
        want = random_brickwork(n, depth, seed).to_ops()
        for uni in (reference.uniforms, oracle.uniforms):
            got = brickwork_ops(n, depth, seed, uni)
            assert got.tobytes() == want.tobytes()


def test_reference_timed_run_returns_kets_state(reference, oracle):
    from oracle.oracle import brickwork_ops
    ops = brickwork_ops(8, 6, 5, oracle.uniforms)
    secs, st = reference.run_timed_state(8, ops)
    assert secs >= 0.0
    assert np.array_equal(st, reference.run(8, ops))


@pytest.mark.parametrize("k", [4, 5, 6])
def test_band_ordered_plans_apply_the_same_circuit(oracle, k):
    """The greedy planner grows blocks over the program order and over band
    orders (gates by ASAP depth band, then lowest qubit, under every
    dependency) and keeps the cheapest partition.  The passes' gate lists,
    concatenated, must be a reordering of the circuit that the FP64 oracle
    evaluates to the same state, with every gate exactly once."""
    import ket_b200 as ket
    from ket_b200.api import Plan
    from ket_b200.workloads import qft_ghz_rz, random_brickwork, random_mixed
    for c in (random_brickwork(12, 12, seed=4), random_mixed(11, 10, seed=6), qft_ghz_rz(10, seed=2)):
        n = c.n_qubits
        ops = c.to_ops()
        p = Plan(n, ops, ket.make_options("c64", "greedy", k, True))
        order = []
        for i in range(p.stats()["n_passes"]):
            order += p.pass_gates(i)
        assert sorted(order) == list(range(len(ops)))
        want = oracle.run(n, ops, fuse=0)
        got = oracle.run(n, ops[np.array(order)].copy(), fuse=0)
        assert np.abs(got - want).max() < 1e-12


def test_band_orders_cut_the_brick_wall_passes():
    """30 qubits x 40 layers: 154 passes in program order at k = 5, 119 with
    the band orders (every width 3..8 at every offset); at k = 6, 65."""
    import ket_b200 as ket
    from ket_b200.workloads import random_brickwork
    c = random_brickwork(30, 40)
    assert ket.plan_stats(c, ket.make_options("c64", "greedy", 5, True))["n_passes"] == 119
    assert ket.plan_stats(c, ket.make_options("c64", "greedy", 6, True))["n_passes"] == 65


def test_six_qubit_blocks_copy_half_tiles():
    """k = 6 blocks whose qubit 0 is a group bit fetch each tile as two tensor
    copies of half a tile (split by the highest target), so three 32 KB
    staging slots fit beside the 128 KB of B images; blocks on qubit 0 keep
    the single 64 KB cp.async slot."""
    import collections
    import ket_b200 as ket
    from ket_b200.api import Plan
    from ket_b200.workloads import random_brickwork
    p = Plan(30, random_brickwork(30, 40).to_ops(), ket.make_options("c64", "greedy", 6, True))
    forms = collections.Counter()
    for i in range(p.stats()["n_passes"]):
        info = p.pass_info(i)
        if info["kind"] == 2 and info["tensor"]:
            f = p.pass_tc_form(i)
            forms[(info["k"], f["tma_dims"] > 0, f["direct"])] += 1
    assert forms == {(6, True, True): 56, (6, False, False): 7}
    for qs, want in {(2, 3, 4, 5, 6, 7): 3, (1, 3, 5, 7, 9, 11): 3, (10, 11, 12, 13, 14, 15): 3,
                     (0, 1, 2, 3, 4, 5): 0}.items():
        c = ket.Circuit(28)
        for q in qs:
            c.u(q, 0.3, 0.2, 0.1)
        for a, b in zip(qs[:-1], qs[1:]):
            c.cx(a, b)
        pp = Plan(28, c.to_ops(), ket.make_options("c64", "greedy", 6, True))
        tc = [i for i in range(pp.stats()["n_passes"]) if pp.pass_info(i)["tensor"]]
        assert pp.pass_tc_form(tc[0])["tma_dims"] == want, qs


@pytest.mark.parametrize("k", [4, 5, 6])
def test_tensor_core_b_image_split_and_layout(k):
    """The B operand plans upload for a tensor-core block, built on the
    host: B[kk][n] = real embedding of the block matrix (B[2c][2r] = Re M[r][c],
    B[2c+1][2r] = -Im M, B[2c][2r+1] = Im M, B[2c+1][2r+1] = Re M), scaled by
    2^sb with its largest entry in [2^14, 2^15); hi = fp16(x) and lo =
    fp16(x - hi), both rounded to nearest even (numpy's float16 is the
    reference), at the K-major 128-byte-swizzle offset of (row n, column kk)
    in whole 128-byte atoms along K; sb last."""
    from ket_b200 import _lib
    dim = 1 << k
    K = N = 2 * dim
    rng = np.random.default_rng(k)
    q, _ = np.linalg.qr(rng.standard_normal((dim, dim)) + 1j * rng.standard_normal((dim, dim)))
    m = np.ascontiguousarray(q, dtype=np.complex128)
    words = ct.c_uint64()
    assert _lib.lib.ketgpu_tc_image(k, m.ctypes.data, None, 0, ct.byref(words)) == 0
    out = np.zeros(words.value, dtype=np.uint32)
    assert _lib.lib.ketgpu_tc_image(k, m.ctypes.data, out.ctypes.data, out.size, ct.byref(words)) == 0
    img = (K + 63) // 64 * N * 128  # bytes per image
    assert words.value * 4 == 2 * img + 16
    raw = out.view(np.uint8)
    hi = raw[:img].view(np.uint16)
    lo = raw[img:2 * img].view(np.uint16)
    sb = int(out[2 * img // 4].view(np.int32))
    B = np.zeros((K, N))
    B[0::2, 0::2] = m.real.T
    B[1::2, 0::2] = -m.imag.T
    B[0::2, 1::2] = m.imag.T
    B[1::2, 1::2] = m.real.T
    assert 2.0 ** 14 <= np.abs(B).max() * 2.0 ** sb < 2.0 ** 15
    kk, n = np.meshgrid(np.arange(K), np.arange(N), indexing="ij")
    off = (kk >> 6) * N * 128 + n * 128 + ((((kk & 63) >> 3) ^ (n & 7)) << 4) + (kk & 7) * 2
    v = np.ldexp(B, sb)
    h = v.astype(np.float16)
    l_ = (v - h.astype(np.float64)).astype(np.float16)
    assert np.array_equal(hi[off // 2], h.view(np.uint16))
    assert np.array_equal(lo[off // 2], l_.view(np.uint16))
    # every used 16-bit slot is addressed once; at k = 4 half of each atom row is unused
    assert len(np.unique(off)) == K * N
    # what the MMAs sum: hi + lo within 2^-22 of each scaled entry's magnitude
    # (plus fp16's subnormal spacing for tiny entries)
    err = np.abs(h.astype(np.float64) + l_.astype(np.float64) - v)
    assert np.all(err <= np.abs(v) * 2.0 ** -22 + 2.0 ** -25)
    assert _lib.lib.ketgpu_tc_image(3, m.ctypes.data, None, 0, ct.byref(words)) != 0


def test_norm_passes_around_tensor_core_blocks():
    """Plans with tensor-core blocks capture the norm first and restore it
    last; when the last block is on the tensor cores it sums the norm as it
    stores, so the restore moves 2 x the state (rescale) instead of 3 x
    (norm read + rescale).  SIMT plans asked to renormalize keep the read."""
    import ket_b200 as ket
    from ket_b200.api import Plan
    from ket_b200.workloads import random_brickwork
    n = 20
    ops = random_brickwork(n, 10).to_ops()
    state = 8 * 2.0 ** n
    p = Plan(n, ops, ket.make_options("c64", "greedy", 6, True))
    kinds = [p.pass_info(i) for i in range(int(p.stats()["n_passes"]))]
    assert kinds[0]["kind"] == 3 and kinds[-1]["kind"] == 3
    assert kinds[-2]["kind"] == 2 and kinds[-2]["tensor"]
    assert kinds[0]["bytes"] == state and kinds[-1]["bytes"] == 2 * state
    q = Plan(n, ops, ket.make_options("c64", "greedy", 5, False, renormalize=1))
    kq = [q.pass_info(i) for i in range(int(q.stats()["n_passes"]))]
    assert kq[0]["kind"] == 3 and kq[-1]["kind"] == 3 and not kq[-2]["tensor"]
    assert kq[-1]["bytes"] == 3 * state
    r = Plan(n, ops, ket.make_options("c64", "greedy", 5, False))
    assert all(r.pass_info(i)["kind"] != 3 for i in range(int(r.stats()["n_passes"])))


def test_plan_block_matrices_match_the_oracle(oracle, golden):
    """Every dense block's FP64 matrix, as the planner built it (on host
    threads, after partitioning), equals the oracle's product of the block's
    gates; the plans are rebuilt many times, so a matrix written by the
    wrong job or a race between the builders would show up."""
    import ctypes as ct
    import ket_b200 as ket
    from ket_b200 import _lib
    from ket_b200.api import Plan
    from ket_b200.workloads import random_brickwork, random_mixed
    g = golden("random_mixed")
    cases = [(n, g[f"ops_{n}"]) for n in (6, 10, 12)]
    cases += [(14, random_mixed(14, 12, seed=4).to_ops()), (20, random_brickwork(20, 12, seed=7).to_ops())]
    for rep in range(20):
        for n, ops in cases:
            for prec, k, tc in (("c128", 5, True), ("c64", 6, True), ("c128", 3, True), ("c64", 4, False)):
                p = Plan(n, ops, ket.make_options(prec, "greedy", k, tc))
                for i in range(int(p.stats()["n_passes"])):
                    if p.pass_info(i)["kind"] != 2:
                        continue
                    qs = p.pass_qubits(i)
                    gates = p.pass_gates(i)
                    cnt = ct.c_uint64()
                    buf = np.zeros(2 << (2 * len(qs)))
                    assert _lib.lib.ketgpu_plan_pass_matrix(p._h, i, buf.ctypes.data, buf.size, ct.byref(cnt)) == 0
                    got = buf.view(np.complex128).reshape(1 << len(qs), 1 << len(qs))
                    want = oracle.block_matrix(np.ascontiguousarray(ops[gates]), qs)
                    assert np.abs(got - want).max() < 1e-12, (rep, n, prec, k, i)
                p.close()
