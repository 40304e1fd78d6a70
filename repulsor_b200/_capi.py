"""ctypes binding of ``librepulsor_b200.so`` (declared in ``include/repulsor_b200.h``).

The library is built in-tree (``make -C repulsor_b200``). There is no CPU
fallback: loading fails loudly when the shared object is missing, and the first
mesh creation fails with ``RPB_ECUDA`` when no CUDA device is present.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librepulsor_b200.so")

RPB_OK, RPB_EINVAL, RPB_ENOTCONV, RPB_ESTALL, RPB_ECUDA, RPB_ENOMEM, RPB_ETIMEOUT = range(7)
STATUS_NAMES = {0: "RPB_OK", 1: "RPB_EINVAL", 2: "RPB_ENOTCONV", 3: "RPB_ESTALL", 4: "RPB_ECUDA",
                5: "RPB_ENOMEM", 6: "RPB_ETIMEOUT"}

PRECOND_NONE, PRECOND_REFERENCE, PRECOND_LEARNED, PRECOND_HYBRID = 0, 1, 2, 3

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_int64)
_fp = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p


class Settings(ctypes.Structure):
    _fields_ = [("split_threshold", ctypes.c_int),
                ("far_field_separation", ctypes.c_double),
                ("near_field_separation", ctypes.c_double),
                ("near_field_intersection", ctypes.c_double),
                ("max_refinement", ctypes.c_int),
                ("thread_count", ctypes.c_int),
                ("device", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("vertex_count", ctypes.c_int64),
                ("simplex_count", ctypes.c_int64),
                ("cluster_count", ctypes.c_int64),
                ("tree_depth", ctypes.c_int64),
                ("near_nnz", ctypes.c_int64),
                ("far_nnz", ctypes.c_int64),
                ("verynear_nnz", ctypes.c_int64),
                ("inter_nnz", ctypes.c_int64),
                ("tree_build_seconds", ctypes.c_double),
                ("device_bytes", ctypes.c_int64)]


class SolveInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int),
                ("restarts", ctypes.c_int),
                ("fallback_iteration", ctypes.c_int),
                ("supernode_levels", ctypes.c_int),
                ("factor_seconds", ctypes.c_double),
                ("factor_nnz", ctypes.c_int64),
                ("factor_on_device", ctypes.c_int)]


# name -> (restype, argtypes); every exported symbol of include/repulsor_b200.h
SIGNATURES = {
    "rpb_default_settings": (ctypes.c_int, [ctypes.POINTER(Settings)]),
    "rpb_last_error": (ctypes.c_char_p, []),
    "rpb_mesh_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int64, _ip, ctypes.c_int64, _dp,
                                       ctypes.POINTER(Settings), ctypes.POINTER(_vp)]),
    "rpb_mesh_destroy": (ctypes.c_int, [_vp]),
    "rpb_mesh_stats": (ctypes.c_int, [_vp, ctypes.POINTER(Stats)]),
    "rpb_mesh_build_info": (ctypes.c_int, [_vp, _ip, _ip]),
    "rpb_mesh_set_stream": (ctypes.c_int, [_vp, _vp]),
    "rpb_mesh_get_stream": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "rpb_mesh_semistatic_update": (ctypes.c_int, [_vp, _dp, ctypes.c_int]),
    "rpb_mesh_semistatic_update_device": (ctypes.c_int, [_vp, _vp]),
    "rpb_mesh_tree": (ctypes.c_int, [_vp, _ip, _ip, _ip, _ip, _ip]),
    "rpb_mesh_pattern": (ctypes.c_int, [_vp, ctypes.c_int, _lp, _ip]),
    "rpb_tree_build_host": (ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_int64, _ip, ctypes.c_int64,
                                           ctypes.POINTER(Settings), ctypes.POINTER(_vp)]),
    "rpb_tree_host_stats": (ctypes.c_int, [_vp, ctypes.POINTER(Stats)]),
    "rpb_tree_host_arrays": (ctypes.c_int, [_vp, _ip, _ip, _ip, _ip, _ip]),
    "rpb_tree_host_pattern": (ctypes.c_int, [_vp, ctypes.c_int, _lp, _ip]),
    "rpb_tree_host_destroy": (ctypes.c_int, [_vp]),
    "rpb_tree_host_obstacle_pattern": (ctypes.c_int, [_vp, _dp, _ip, _vp, _dp, _ip, ctypes.c_int, _lp, _lp, _ip]),
    "rpb_h1_solve_host": (ctypes.c_int, [_vp, _dp, _ip, _dp, _dp, ctypes.c_int]),
    "rpb_tpe0_value": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, _dp]),
    "rpb_tpe0_differential": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, _dp, ctypes.c_int, _dp]),
    "rpb_tpe0_differential_device": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                    ctypes.c_double, _vp, ctypes.c_int, _dp]),
    "rpb_tpm0_multiply": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, ctypes.c_int,
                                         ctypes.c_double, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "rpb_tpm0_multiply_device": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, _vp,
                                                ctypes.c_int, ctypes.c_double, _vp, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int]),
    "rpb_tpm0_precondition": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp,
                                             ctypes.c_int, ctypes.c_double, _dp, ctypes.c_int, ctypes.c_int]),
    "rpb_tpm0_solve": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, ctypes.c_int,
                                      ctypes.c_double, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_double, ctypes.c_int, _ip, _dp]),
    "rpb_tpe0_stage_times": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int64,
                                            _dp]),
    "rpb_measure_fp32_peak": (ctypes.c_int, [ctypes.c_int, _dp]),
    "rpb_tpe0_value_noalloc": (ctypes.c_int, [ctypes.c_int, _vp, ctypes.c_int64, _vp, ctypes.c_int64, _vp, _vp, _vp,
                                              ctypes.c_int64, _vp, _vp, _vp, _vp, ctypes.c_int64, ctypes.c_double,
                                              ctypes.c_double, _vp, _vp]),
    "rpb_tpm0_solve_info": (ctypes.c_int, [_vp, ctypes.POINTER(SolveInfo)]),
    "rpb_tpe0_energy_device": (ctypes.c_int, [_vp, _vp]),
    "rpb_mesh_maximum_safe_step_size": (ctypes.c_int, [_vp, _dp, ctypes.c_double, ctypes.c_double, _dp]),
    "rpb_mesh_set_shards": (ctypes.c_int, [_vp, ctypes.c_int]),
    "rpb_mesh_shard_rows": (ctypes.c_int, [_vp, ctypes.c_int, _lp, _lp]),
    "rpb_mesh_shard_buffer_doubles": (ctypes.c_int, [_vp, _lp]),
    "rpb_tpe0_pairs_shard": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, _vp]),
    "rpb_tpe0_collect_shards": (ctypes.c_int, [_vp, _vp, ctypes.c_double, ctypes.c_double, _vp, ctypes.c_int]),
    "rpb_tpe0_simplex_densities": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, _dp, _dp]),
    "rpb_tpe0_vertex_densities": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, _dp, _dp]),
    "rpb_mesh_load_obstacle": (ctypes.c_int, [_vp, _vp]),
    "rpb_mesh_obstacle_stats": (ctypes.c_int, [_vp, _lp]),
    "rpb_mesh_obstacle_pattern": (ctypes.c_int, [_vp, ctypes.c_int, _lp, _ip]),
    "rpb_tpoe_value": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, _dp]),
    "rpb_tpoe_differential": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             _dp, ctypes.c_int, _dp]),
    "rpb_tpoe_differential_device": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                    ctypes.c_double, _vp, ctypes.c_int, _dp]),
    "rpb_mlp_param_count": (ctypes.c_int, []),
    "rpb_mlp_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(_vp)]),
    "rpb_mlp_destroy": (ctypes.c_int, [_vp]),
    "rpb_mlp_get_params": (ctypes.c_int, [_vp, _fp]),
    "rpb_mlp_set_params": (ctypes.c_int, [_vp, _fp]),
    "rpb_mlp_eval": (ctypes.c_int, [_vp, _fp, ctypes.c_int64, _fp, _fp, _fp]),
    "rpb_mlp_train_step": (ctypes.c_int, [_vp, _vp, ctypes.c_double, ctypes.c_double, _dp, _dp, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_double, _dp, _fp]),
    "rpb_mesh_set_learned": (ctypes.c_int, [_vp, _vp]),
    "rpb_tpm0_learned_apply": (ctypes.c_int, [_vp, _dp, _dp]),
    "rpb_tpm0_learned_apply_pair": (ctypes.c_int, [_vp, _dp, _dp, _dp, _dp]),
    "rpb_mlp_train_step_sens": (ctypes.c_int, [_vp, _vp, _dp, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                               _dp, ctypes.POINTER(ctypes.c_float)]),
}

_lib = None


def load():
    """Load the shared library (raises OSError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} not found: build it with `make -C repulsor_b200` (no CPU fallback exists)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class RepulsorError(RuntimeError):
    def __init__(self, status, where):
        msg = load().rpb_last_error().decode(errors="replace")
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def check(status, where):
    if status != RPB_OK:
        raise RepulsorError(status, where)


def dptr(a):
    return a.ctypes.data_as(_dp)


def iptr(a):
    return a.ctypes.data_as(_ip)


def lptr(a):
    return a.ctypes.data_as(_lp)


def fptr(a):
    return a.ctypes.data_as(_fp)
