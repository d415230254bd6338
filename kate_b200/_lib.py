"""Loads libkate_b200.so (built in-tree by kate_b200/build.py) and declares
the C ABI of include/kate_b200.h for ctypes. There is no fallback: if the
library is missing the import fails loudly."""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkate_b200.so")

_lib = None

_c = ctypes
_i, _d, _vp = _c.c_int, _c.c_double, _c.c_void_p
_ip, _dp = _c.POINTER(_c.c_int), _c.POINTER(_c.c_double)
_u64, _u64p = _c.c_uint64, _c.POINTER(_c.c_uint64)
_vpp = _c.POINTER(_c.c_void_p)

# name -> argtypes (every function returns kate_status unless listed in _RET)
SIGNATURES = {
    "kate_last_error": [],
    "kate_version": [],
    "kate_device_count": [_ip],
    "kate_device_properties": [_i, _c.c_char_p, _i, _c.POINTER(_c.c_size_t), _c.POINTER(_c.c_size_t), _ip],
    "kate_circuit_create": [_i, _vpp],
    "kate_circuit_destroy": [_vp],
    "kate_circuit_clone": [_vp, _vpp],
    "kate_circuit_nqbits": [_vp, _ip],
    "kate_circuit_append_gate": [_vp, _i, _ip, _i, _i],
    "kate_circuit_append_dense": [_vp, _dp, _ip, _i],
    "kate_circuit_append_many": [_vp, _i, _ip, _ip, _ip, _ip, _dp],
    "kate_circuit_num_gates": [_vp, _ip],
    "kate_circuit_get_gate": [_vp, _i, _ip, _ip, _ip, _ip, _dp],
    "kate_circuit_schedule": [_vp],
    "kate_circuit_fuse": [_vp, _i, _d],
    "kate_circuit_group": [_vp, _i],
    "kate_circuit_allocate": [_vp, _i, _i],
    "kate_circuit_compile_default": [_vp, _i, _i],
    "kate_circuit_compile_opt": [_vp, _i, _d, _i, _i, _i],
    "kate_circuit_num_groups": [_vp, _ip],
    "kate_circuit_get_group": [_vp, _i, _ip, _ip, _ip],
    "kate_circuit_num_instructions": [_vp, _ip],
    "kate_circuit_get_instruction": [_vp, _i, _ip, _ip, _ip],
    "kate_circuit_get_permutations": [_vp, _ip, _ip, _ip],
    "kate_merge_gates": [_vp, _i, _i, _ip, _ip, _dp],
    "kate_merge_gates_device": [_vp, _i, _i, _i, _vp, _ip, _ip, _dp],
    "kate_circuit_fuse_device": [_vp, _i, _d, _i],
    "kate_circuit_export_qcx": [_vp, _c.c_char_p],
    "kate_sim_create": [_vp, _i, _i, _vpp],
    "kate_sim_destroy": [_vp],
    "kate_sim_execute": [_vp, _dp],
    "kate_sim_execute_from": [_vp, _dp, _dp],
    "kate_sim_execute_timed": [_vp, _dp, _dp, _dp],
    "kate_sim_run_async": [_vp, _vp],
    "kate_sim_synchronize": [_vp],
    "kate_sim_proba_state": [_vp, _dp],
    "kate_sim_get_state": [_vp, _dp],
    "kate_sim_set_state": [_vp, _dp],
    "kate_sim_expect_z": [_vp, _dp],
    "kate_sim_probabilities": [_vp, _dp],
    "kate_sim_sample": [_vp, _i, _u64, _u64p],
    "kate_sim_state_device": [_vp, _vpp, _ip],
    "kate_sim_nqbits": [_vp, _ip],
    "kate_sim_profile_passes": [_vp, _c.POINTER(_c.c_float), _c.POINTER(_c.c_float)],
    "kate_sim_launches_per_run": [_vp, _ip],
    "kate_sim_pass_kernel": [_vp, _i, _ip],
    "kate_sim_pass_work": [_vp, _i, _c.POINTER(_c.c_double)],
    "kate_batch_get_state": [_vp, _i, _dp],
    "kate_sim_norm2_before_renorm": [_vp, _dp],
    "kate_sim_num_passes": [_vp, _ip],
    "kate_sim_get_pass": [_vp, _i, _ip, _ip, _ip],
    "kate_plan_create": [_vp, _i, _i, _c.c_uint, _vpp],
    "kate_plan_destroy": [_vp],
    "kate_plan_num_passes": [_vp, _ip],
    "kate_plan_get_pass": [_vp, _i, _ip, _c.POINTER(_c.c_uint8), _c.POINTER(_c.c_uint8)],
    "kate_plan_num_ops": [_vp, _ip],
    "kate_plan_get_op": [_vp, _i, _ip, _u64p, _dp],
    "kate_plan_final_layout": [_vp, _ip, _ip],
    "kate_plan_get_program": [_vp, _i, _vp, _c.c_size_t, _c.POINTER(_c.c_size_t), _ip],
    "kate_plan_pass_source": [_vp, _i, _i, _c.c_char_p, _c.c_size_t, _c.POINTER(_c.c_size_t)],
    "kate_plan_num_smem_ops": [_vp, _ip],
    "kate_plan_get_block_program": [_vp, _i, _vp, _c.c_size_t, _c.POINTER(_c.c_size_t), _ip],
    "kate_plan_block_images": [_vp, _vp, _c.c_size_t, _c.POINTER(_c.c_size_t)],
    "kate_plan_get_smem_op": [_vp, _i, _ip, _u64p, _dp],
    "kate_proba_state_noalloc": [_vp, _c.c_size_t, _i, _ip, _ip, _dp, _vp],
    "kate_batch_options_default": [_vp],
    "kate_batch_autotune": [_vpp, _i, _i, _i, _vp],
    "kate_batch_create": [_vpp, _i, _i, _i, _vp, _vpp],
    "kate_batch_destroy": [_vp],
    "kate_batch_run_async": [_vp, _vp],
    "kate_batch_synchronize": [_vp],
    "kate_batch_run": [_vp],
    "kate_batch_expect_z": [_vp, _dp],
    "kate_batch_num_outputs": [_vp, _c.POINTER(_c.c_longlong)],
    "kate_batch_info": [_vp, _c.POINTER(_c.c_longlong)],
    "kate_batch_block_programs": [_vp, _c.POINTER(_c.c_longlong)],
    "kate_batch_time": [_vp, _i, _c.POINTER(_c.c_float)],
    "kate_batch_circuit_info": [_vp, _ip, _ip],
    "kate_batch_create_times": [_vp, _dp],
    "kate_release_cached_memory": [_i],
    "kate_batch_upload_bytes": [_vp, _c.POINTER(_c.c_longlong)],
    "kate_server_options_default": [_vp],
    "kate_server_create": [_i, _i, _vp, _vpp],
    "kate_server_destroy": [_vp],
    "kate_server_submit": [_vp, _vp, _i, _u64, _c.POINTER(_c.c_longlong)],
    "kate_server_wait": [_vp, _c.c_longlong, _d, _ip, _dp, _u64p, _dp],
    "kate_server_stats": [_vp, _c.POINTER(_c.c_longlong)],
    "kate_server_now": [_vp, _dp],
}

KATE_BATCH_MAX_QUBITS = 28


class BatchTuning(_c.Structure):
    _fields_ = [("fusion", _c.c_int), ("max_gates", _c.c_int), ("group_qubits", _c.c_int), ("coalesce", _c.c_int),
                ("blocks", _c.c_int)]


class BatchOptions(_c.Structure):
    """kate_batch_options (include/kate_b200.h)."""
    _fields_ = [("chunk", _c.c_int), ("zchunks", _c.c_int), ("window_bytes", _c.c_ulonglong),
                ("tune", BatchTuning * (KATE_BATCH_MAX_QUBITS + 1)), ("wait_ms", _c.c_int),
                ("fault_task", _c.c_longlong)]
_RET = {"kate_last_error": _c.c_char_p, "kate_version": _c.c_char_p}


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m kate_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _RET.get(name, _i)
        _lib = L
    return _lib


def last_error() -> str:
    return lib().kate_last_error().decode(errors="replace")


class ServerOptions(_c.Structure):
    """kate_server_options (include/kate_b200.h)."""
    _fields_ = [("budget_bytes", _c.c_ulonglong), ("aux_bytes", _c.c_ulonglong), ("step_tiles", _c.c_longlong),
                ("chunk", _c.c_int), ("zchunks", _c.c_int), ("schunks", _c.c_int), ("planners", _c.c_int),
                ("fusion", _c.c_int), ("max_gates", _c.c_int), ("step_latency_us", _c.c_int),
                ("tensor_blocks", _c.c_int)]
