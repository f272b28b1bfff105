"""ketgpu_expval_sum_noalloc: the Pauli-sum expectation for callers that
cannot allocate device memory during the call (a service keeping nearly all
of HBM reserved for resident states, or code that must not have device
memory allocated and freed underneath it).  Called through the C ABI, it
must give ketgpu_expval_sum's value -- on two calls in a row, since every
call reuses the same fixed scratch array -- and refuse more terms than that
array holds.  Collected last on purpose: it runs after every other test, and
also passes alone in a fresh process."""
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
