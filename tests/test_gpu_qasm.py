"""OpenQASM programs run on the GPU: the states of ket_b200.from_qasm's
circuits against ket::run's (tests/golden/qasm.json), complex128 at 1e-12
max-abs per amplitude (ket's own tolerance, tests/test_simulator.cpp:9) and
complex64 at 1e-5."""
import json
import os

import numpy as np
import pytest

import ket_b200 as ket

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "qasm.json")


def _cases():
    with open(GOLDEN) as f:
        progs = json.load(f)["programs"]
    return [p for p in progs if "state" in p]


@pytest.mark.parametrize("precision,tol", [("c128", 1e-12), ("c64", 1e-5)])
def test_qasm_programs_run_like_ket(precision, tol):
    try:
        for fusion in ("none", "greedy"):
            ket.set_options(precision=precision, fusion=fusion)
            for prog in _cases():
                want = np.array([complex(float.fromhex(a), float.fromhex(b)) for a, b in prog["state"]])
                got = ket.run(ket.from_qasm(prog["source"])).to_numpy()
                assert np.abs(got - want).max() < tol, (prog["name"], precision, fusion)
    finally:
        ket.set_options(precision="c128", fusion="greedy")
