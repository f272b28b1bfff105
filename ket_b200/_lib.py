"""ctypes binding of libket_b200.so (the C ABI in include/ket_b200.h).

The library is loaded from the package directory only.  If it is missing or
cannot be loaded the import fails loudly: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libket_b200.so")

OK = 0
ERR_OUT_OF_RANGE = -1
ERR_INVALID = -2
ERR_LOGIC = -3
ERR_CUDA = -4
ERR_OOM = -5
ERR_TIMEOUT = -6

C64, C128 = 0, 1
FUSE_NONE, FUSE_REFERENCE, FUSE_GREEDY, FUSE_LEARNED = 0, 1, 2, 3

# ketgpu_op: 48 bytes, identical to the C struct.
OP_DTYPE = np.dtype([("type", "<i4"), ("nq", "<i4"), ("q", "<i4", (3,)),
                     ("aux", "<i4"), ("p", "<f8", (3,))], align=True)
assert OP_DTYPE.itemsize == 48


class Options(ct.Structure):
    _fields_ = [("precision", ct.c_int32), ("fusion", ct.c_int32),
                ("max_block_qubits", ct.c_int32), ("tensor_cores", ct.c_int32),
                ("renormalize", ct.c_int32)]


class PlanStats(ct.Structure):
    _fields_ = [("n_gates", ct.c_uint64), ("n_passes", ct.c_uint64), ("n_fused", ct.c_uint64),
                ("n_tensor", ct.c_uint64), ("bytes", ct.c_double), ("flops", ct.c_double),
                ("predicted_us", ct.c_double)]


class KetGpuError(RuntimeError):
    pass


class KetGpuTimeout(KetGpuError):
    pass


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"ket_b200: {LIB_PATH} is missing; build it with `python ket_b200/build.py` "
            "(the backend has no CPU fallback)")
    L = ct.CDLL(LIB_PATH)
    vp, sz, i32, u32, u64 = ct.c_void_p, ct.c_size_t, ct.c_int32, ct.c_uint32, ct.c_uint64
    pd = ct.POINTER(ct.c_double)
    sig = {
        "ketgpu_last_error": ([], ct.c_char_p),
        "ketgpu_abi_version": ([], ct.c_int),
        "ketgpu_launch_count": ([], u64),
        "ketgpu_state_create": ([i32, i32, ct.POINTER(vp)], ct.c_int),
        "ketgpu_state_destroy": ([vp], ct.c_int),
        "ketgpu_state_reset": ([vp], ct.c_int),
        "ketgpu_state_info": ([vp, ct.POINTER(i32), ct.POINTER(i32)], ct.c_int),
        "ketgpu_state_device_ptr": ([vp], vp),
        "ketgpu_state_download": ([vp, u64, u64, vp], ct.c_int),
        "ketgpu_state_upload": ([vp, u64, u64, vp], ct.c_int),
        "ketgpu_state_download_raw": ([vp, u64, u64, vp], ct.c_int),
        "ketgpu_state_copy": ([vp, vp], ct.c_int),
        "ketgpu_state_synchronize": ([vp], ct.c_int),
        "ketgpu_plan_create": ([i32, vp, u64, ct.POINTER(Options), ct.POINTER(vp)], ct.c_int),
        "ketgpu_plan_destroy": ([vp], ct.c_int),
        "ketgpu_plan_stats_get": ([vp, ct.POINTER(PlanStats)], ct.c_int),
        "ketgpu_plan_execute": ([vp, vp], ct.c_int),
        "ketgpu_plan_execute_timed": ([vp, vp, vp], ct.c_int),
        "ketgpu_plan_pass_info": ([vp, u64, ct.POINTER(i32), ct.POINTER(i32), ct.POINTER(i32), pd], ct.c_int),
        "ketgpu_plan_pass_qubits": ([vp, u64, ct.POINTER(i32), i32, ct.POINTER(i32)], ct.c_int),
        "ketgpu_plan_pass_gates": ([vp, u64, ct.POINTER(i32), i32, ct.POINTER(i32)], ct.c_int),
        "ketgpu_release_cache": ([], ct.c_int),
        "ketgpu_run_last_profile": ([vp], ct.c_int),
        "ketgpu_plan_pass_tc_form": ([vp, u64, ct.POINTER(i32), ct.POINTER(i32)], ct.c_int),
        "ketgpu_tc_image": ([i32, vp, vp, u64, ct.POINTER(u64)], ct.c_int),
        "ketgpu_plan_pass_matrix": ([vp, u64, vp, u64, ct.POINTER(u64)], ct.c_int),
        "ketgpu_state_stream": ([vp], vp),
        "ketgpu_apply": ([vp, vp, u64, ct.POINTER(Options)], ct.c_int),
        "ketgpu_run": ([i32, vp, u64, ct.POINTER(Options), vp], ct.c_int),
        "ketgpu_norm": ([vp, pd], ct.c_int),
        "ketgpu_inner": ([vp, vp, pd, pd], ct.c_int),
        "ketgpu_compare": ([vp, vp, vp], ct.c_int),
        "ketgpu_expval": ([vp, ct.c_char_p, pd], ct.c_int),
        "ketgpu_expval_sum": ([vp, vp, vp, u64, pd], ct.c_int),
        "ketgpu_expval_terms": ([vp, vp, u64, vp], ct.c_int),
        "ketgpu_expval_sum_noalloc": ([vp, vp, vp, u64, pd], ct.c_int),
        "ketgpu_uniforms_mt19937": ([u32, u64, vp], ct.c_int),
        "ketgpu_sample": ([vp, vp, u64, vp], ct.c_int),
        "ketgpu_measure": ([vp, u32, ct.POINTER(u64)], ct.c_int),
        "ketgpu_sample_seeded": ([vp, u32, u64, vp], ct.c_int),
        "ketgpu_sample_tree_builds": ([], u64),
        "ketgpu_adjoint": ([i32, vp, u64, vp, vp, u64, u64, vp, vp, u64, i32, i32, vp, vp], ct.c_int),
        "ketgpu_adjoint_ex": ([i32, vp, u64, vp, vp, u64, u64, vp, vp, u64, i32, i32, i32, vp, vp], ct.c_int),
        "ketgpu_adjoint_plan_describe": ([i32, vp, u64, vp, i32, i32, vp, u64, vp], ct.c_int),
        "ketgpu_adjoint_jit_info": ([vp, vp, vp], ct.c_int),
        "ketgpu_mlp_create": ([u64, ct.POINTER(vp)], ct.c_int),
        "ketgpu_mlp_destroy": ([vp], ct.c_int),
        "ketgpu_mlp_get_weights": ([vp] * 7, ct.c_int),
        "ketgpu_mlp_set_weights": ([vp] * 7, ct.c_int),
        "ketgpu_mlp_forward": ([vp, vp, u64, vp], ct.c_int),
        "ketgpu_mlp_gradients": ([vp, vp, vp, u64] + [vp] * 7, ct.c_int),
        "ketgpu_mlp_train": ([vp, vp, vp, u64, u64, u64, ct.c_float, vp], ct.c_int),
        "ketgpu_planner_set_model": ([vp], ct.c_int),
        "ketgpu_block_features": ([i32, i32, vp, u64, i32, i32, vp], ct.c_int),
        "ketgpu_plan_pass_features": ([vp, u64, vp], ct.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    return L


lib = _load()


def check(rc: int) -> None:
    """Raise the exception ket would have thrown for a KETGPU_ERR_* code."""
    if rc == OK:
        return
    msg = lib.ketgpu_last_error().decode(errors="replace")
    if rc == ERR_OUT_OF_RANGE:
        raise IndexError(msg)
    if rc == ERR_INVALID:
        raise ValueError(msg)
    if rc == ERR_OOM:
        raise MemoryError(msg)
    if rc == ERR_TIMEOUT:
        raise KetGpuTimeout(msg)
    raise KetGpuError(f"{msg} (code {rc})")


def c_strings(strings):
    """Keep-alive pair (array of char*, buffers) for a list of Python strings."""
    bufs = [ct.create_string_buffer(s.encode()) for s in strings]
    arr = (ct.c_char_p * max(1, len(bufs)))(*[ct.cast(b, ct.c_char_p) for b in bufs])
    return arr, bufs


def launch_count() -> int:
    return int(lib.ketgpu_launch_count())
