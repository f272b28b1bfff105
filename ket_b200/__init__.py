"""ket_b200 -- B200-native state-vector backend for ket.

Python mirror of ket's API (bindings/python/ket/__init__.py) over the C ABI
of libket_b200.so; every state-vector computation runs in the CUDA kernels
of ket_b200/csrc.
"""
from .api import (DeviceState, Plan, ProbeRun, State, chosen_method, expval, get_options,
                  is_clifford, make_options, measure, num_threads, plan_stats, run, run_device,
                  run_with_probes, sample, sample_shots, set_num_threads, set_options, uniforms,
                  use_learned_planner)
from .circuit import Circuit, Gate, GateType
from .qasm import from_qasm, to_qasm
from ._lib import launch_count

__all__ = [
    "Circuit", "DeviceState", "Gate", "GateType", "Plan", "ProbeRun", "State", "chosen_method",
    "expval", "from_qasm", "get_options", "is_clifford", "launch_count", "make_options", "measure",
    "num_threads", "plan_stats", "run", "run_device", "run_with_probes", "sample", "sample_shots",
    "set_num_threads", "set_options", "to_qasm", "uniforms", "use_learned_planner",
]
