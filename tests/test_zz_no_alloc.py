"""ketgpu_expval_sum_noalloc: the Pauli-sum expectation for callers that
cannot allocate device memory during the call (a service keeping nearly all
of HBM reserved for resident states, or code that must not have device
memory allocated and freed underneath it).  Called through the C ABI, it
must give ketgpu_expval_sum's value and ket's own value from the golden
fixture -- on two calls in a row, since every call reuses the same fixed
scratch array -- leave free device memory and the default memory pool
untouched, and refuse more terms than that array holds.  Collected last on
purpose: it runs after every other test, and also passes alone in a fresh
process."""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the expectation tolerance of the complex128 tests


def _sum(fn, state, terms):
    from ket_b200 import _lib
    coeffs = np.array([c for c, _ in terms], dtype=np.float64)
    arr, keep = _lib.c_strings([p for _, p in terms])
    out = ct.c_double()
    rc = fn(state.handle, coeffs.ctypes.data, ct.cast(arr, ct.c_void_p), len(terms), ct.byref(out))
    return rc, out.value


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_noalloc_matches_allocating_entry_point(prec):
    import ket_b200 as ket
    from ket_b200 import _lib
    from ket_b200.workloads import random_brickwork, random_pauli_sum
    n = 14
    state = ket.run_device(random_brickwork(n, 6, seed=21), options=ket.make_options(prec, "greedy", 5, True))
    for call, nterms in enumerate((40, 7)):  # two calls in a row, the second smaller
        terms = random_pauli_sum(n, nterms, seed=30 + call)
        rc_a, want = _sum(_lib.lib.ketgpu_expval_sum, state, terms)
        rc_b, got = _sum(_lib.lib.ketgpu_expval_sum_noalloc, state, terms)
        assert rc_a == 0 and rc_b == 0
        assert abs(got - want) < TOL * max(1.0, sum(abs(c) for c, _ in terms))
    state.close()


def test_noalloc_rejects_more_terms_than_its_scratch():
    import ket_b200 as ket
    from ket_b200 import _lib
    state = ket.DeviceState(4, "c128")
    terms = [(1.0, "ZZZZ")] * 257
    rc, _ = _sum(_lib.lib.ketgpu_expval_sum_noalloc, state, terms)
    assert rc == _lib.ERR_INVALID
    assert "at most 256 terms" in _lib.lib.ketgpu_last_error().decode()
    rc, v = _sum(_lib.lib.ketgpu_expval_sum_noalloc, state, [(2.0, "ZZZZ")])
    assert rc == 0 and abs(v - 2.0) < TOL
    state.close()


def test_noalloc_matches_kets_golden_expval(golden):
    """ket's expval(State, PauliSum) on its own 10-qubit state (written by ket,
    tests/golden/make_golden.py): all 40 terms, then the first 7."""
    import ket_b200 as ket
    from ket_b200 import _lib
    g = golden("expval")
    amps = golden("random_mixed")["state_10"]
    state = ket.DeviceState(10, "c128").from_numpy(amps)
    coeffs = g["coeffs"].tolist()
    paulis = [str(p) for p in g["paulis"]]
    for nterms in (40, 7):
        terms = list(zip(coeffs[:nterms], paulis[:nterms]))
        rc, got = _sum(_lib.lib.ketgpu_expval_sum_noalloc, state, terms)
        assert rc == 0
        want = g["total"][0] if nterms == 40 else sum(c * v for c, v in zip(coeffs[:nterms], g["values"][:nterms]))
        assert abs(got - want) < TOL
    state.close()


def _default_pool_usage():
    """(used now, used high-water mark) of the current device's default
    stream-ordered memory pool, through the driver API."""
    import torch
    cu = ct.CDLL("libcuda.so.1")
    dev, pool = ct.c_int(), ct.c_void_p()
    assert cu.cuInit(0) == 0
    assert cu.cuDeviceGet(ct.byref(dev), torch.cuda.current_device()) == 0
    assert cu.cuDeviceGetDefaultMemPool(ct.byref(pool), dev) == 0
    used, high = ct.c_uint64(), ct.c_uint64()
    assert cu.cuMemPoolGetAttribute(pool, 7, ct.byref(used)) == 0   # CU_MEMPOOL_ATTR_USED_MEM_CURRENT
    assert cu.cuMemPoolGetAttribute(pool, 8, ct.byref(high)) == 0   # CU_MEMPOOL_ATTR_USED_MEM_HIGH
    return used.value, high.value, cu, pool


def test_noalloc_allocates_no_device_memory():
    """Free device memory (cudaMemGetInfo) and the default pool's usage,
    including its high-water mark reset before the calls, stay the same over
    six calls, the first call on a fresh state included (the scratch array
    and the kernels are loaded when a state is created, not by the call)."""
    import torch
    import ket_b200 as ket
    from ket_b200 import _lib
    from ket_b200.workloads import random_brickwork, random_pauli_sum
    n = 16
    state = ket.run_device(random_brickwork(n, 4, seed=3), options=ket.make_options("c64", "greedy", 5, True))
    terms = random_pauli_sum(n, 200, seed=8)
    torch.cuda.mem_get_info()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    used0, _, cu, pool = _default_pool_usage()
    zero = ct.c_uint64(0)
    assert cu.cuMemPoolSetAttribute(pool, 8, ct.byref(zero)) == 0  # reset the high-water mark
    vals = []
    for _ in range(6):
        rc, v = _sum(_lib.lib.ketgpu_expval_sum_noalloc, state, terms)
        assert rc == 0
        vals.append(v)
    assert len(set(vals)) == 1
    torch.cuda.synchronize()
    used1, high1, _, _ = _default_pool_usage()
    assert torch.cuda.mem_get_info()[0] == free0
    assert used1 == used0 and high1 <= used0
    state.close()
