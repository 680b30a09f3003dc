"""ctypes binding of ``libpggc_b200.so`` (the C ABI in ``include/pggc.h``).

The library is loaded from the in-tree build directory.  There is no fallback:
if the library is missing or a call fails, an exception is raised.
"""
from __future__ import annotations

import ctypes
import os

from . import build as _build

PGGC_OK, PGGC_ERR_INVALID, PGGC_ERR_CUDA, PGGC_ERR_DEVICE, PGGC_ERR_INTERNAL = 0, 1, 2, 3, 4
W_UNIFORM, W_INT32, W_FLOAT32 = 0, 1, 2
OBJ_MOD, OBJ_WMOD, OBJ_CPM, OBJ_NLCC, OBJ_LCC = 0, 1, 2, 3, 4
MEM_HOST, MEM_DEVICE = 0, 1
METHOD_LOUVAIN, METHOD_LEIDEN, METHOD_LEIDEN_PLUS = 0, 1, 2

LIB_PATH = os.path.join(_build.OUT, "libpggc_b200.so")


class PggcError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"pggc status {status}: {message}")
        self.status = status


class InvalidArgument(PggcError):
    pass


class DeviceError(PggcError):
    pass


class Stats(ctypes.Structure):
    _fields_ = [("levels", ctypes.c_int64), ("total_nnz", ctypes.c_int64), ("sweeps", ctypes.c_int64),
                ("moves", ctypes.c_int64), ("passes", ctypes.c_int64), ("objective", ctypes.c_double),
                ("raw_obj", ctypes.c_double), ("label_count", ctypes.c_int64),
                ("filtered_passes", ctypes.c_int64), ("exact_passes", ctypes.c_int64),
                ("judge_gain", ctypes.c_double), ("fell_back", ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchJob(ctypes.Structure):
    _fields_ = [("graph", ctypes.c_void_p), ("objective", ctypes.c_int), ("lambda_mult", ctypes.c_double),
                ("method", ctypes.c_int), ("ex_iters", ctypes.c_int), ("seed", ctypes.c_uint64),
                ("labels_out", ctypes.c_void_p), ("mem_kind", ctypes.c_int), ("stats", Stats),
                ("status", ctypes.c_int)]


class MemeStats(ctypes.Structure):
    _fields_ = [("objective", ctypes.c_double), ("label_count", ctypes.c_int64), ("offspring", ctypes.c_int64),
                ("replaced", ctypes.c_int64), ("best_initial", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tune(ctypes.Structure):
    _fields_ = [("thread_max_deg", ctypes.c_int), ("warp_max_deg", ctypes.c_int), ("load_factor", ctypes.c_double),
                ("streams", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneTrial(ctypes.Structure):
    _fields_ = [("config", Tune), ("seconds", ctypes.c_double), ("edges_per_s", ctypes.c_double)]


# name -> (restype, argtypes)
_vp, _i64, _ci, _dbl, _u32, _u64, _flt = (ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_uint32, ctypes.c_uint64, ctypes.c_float)
_PP = ctypes.POINTER(ctypes.c_void_p)
_SIGS = {
    "pggc_last_error": (ctypes.c_char_p, []),
    "pggc_version": (ctypes.c_char_p, []),
    "pggc_launch_count": (_u64, []),
    "pggc_debug_set_probe_limit": (_ci, [_vp, _ci]),
    "pggc_profile_enable": (_ci, [_vp, _ci]),
    "pggc_profile_reset": (_ci, [_vp]),
    "pggc_profile_names": (_ci, [_vp, ctypes.c_char_p, _i64, ctypes.POINTER(_i64)]),
    "pggc_profile_read": (_ci, [_vp, ctypes.c_char_p, ctypes.POINTER(_i64), ctypes.POINTER(_dbl),
                               ctypes.POINTER(_dbl)]),
    "pggc_context_create": (_ci, [_ci, _PP]),
    "pggc_context_destroy": (_ci, [_vp]),
    "pggc_context_stream": (_ci, [_vp, _PP]),
    "pggc_graph_create": (_ci, [_vp, _i64, _i64, _vp, _vp, _vp, _ci, _vp, _ci, _ci, _PP]),
    "pggc_graph_destroy": (_ci, [_vp]),
    "pggc_graph_set_vertex_weights": (_ci, [_vp, _vp, _vp, _ci]),
    "pggc_graph_load": (_ci, [_vp, ctypes.c_char_p, _ci, ctypes.POINTER(_ci), _PP]),
    "pggc_graph_from_edges": (_ci, [_vp, _i64, _i64, _vp, _vp, _vp, _ci, _ci, _ci, _PP]),
    "pggc_graph_dims": (_ci, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_ci)]),
    "pggc_graph_read": (_ci, [_vp, _vp, _vp, _vp, _vp, _vp, _ci]),
    "pggc_cluster_data_create": (_ci, [_vp, _vp, _ci, _dbl, _PP]),
    "pggc_cluster_data_destroy": (_ci, [_vp]),
    "pggc_cluster_data_get": (_ci, [_vp, ctypes.POINTER(_dbl), ctypes.POINTER(_dbl), ctypes.POINTER(_dbl),
                                    ctypes.POINTER(_dbl), ctypes.POINTER(_i64)]),
    "pggc_cluster_data_total_deg": (_ci, [_vp, _vp, _vp, _ci]),
    "pggc_cluster_data_set": (_ci, [_vp, _vp, _i64, _vp, _dbl, _ci]),
    "pggc_generate_orderings": (_ci, [_vp, _vp, _vp, _vp, _vp, _ci]),
    "pggc_generate_orderings_noalloc": (_ci, [_vp, _i64, _vp, _vp, _vp, _vp]),
    "pggc_mlp_infer": (_ci, [_vp, _vp, _vp, _i64, _ci, _vp]),
    "pggc_mlp_loss_grad": (_ci, [_vp, _vp, _vp, _vp, _i64, _flt, _ci, _vp, _vp]),
    "pggc_mlp_train": (_ci, [_vp, _vp, _vp, _vp, _i64, _ci, _ci, _ci, _flt, _flt, _u64, _vp]),
    "pggc_filter_log_start": (_ci, [_vp, _i64, _dbl, _u64]),
    "pggc_filter_log_stop": (_ci, [_vp, _vp, _vp, _i64, _ci, ctypes.POINTER(_i64)]),
    "pggc_filter_enable": (_ci, [_vp, _vp, _flt]),
    "pggc_filter_stats": (_ci, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64), _ci]),
    "pggc_filter_scope": (_ci, [_vp, _ci, _ci]),
    "pggc_filter_log_label": (_ci, [_vp, _ci]),
    "pggc_batch_run": (_ci, [_vp, _vp, _i64, _ci]),
    "pggc_tune_set": (_ci, [_vp, ctypes.POINTER(Tune)]),
    "pggc_tune_get": (_ci, [_vp, ctypes.POINTER(Tune)]),
    "pggc_batch_autotune": (_ci, [_vp, _vp, _i64, _vp, _i64, ctypes.POINTER(_i64), ctypes.POINTER(Tune)]),
    "pggc_meme_cluster": (_ci, [_vp, _vp, _ci, _dbl, _ci, _i64, _dbl, _u64, _vp, _ci, ctypes.POINTER(MemeStats)]),
    "pggc_intersect_clusters": (_ci, [_vp, _vp, _vp, _i64, _vp, ctypes.POINTER(_i64), _ci]),
    "pggc_cut_signature": (_ci, [_vp, _vp, _vp, _vp, _ci]),
    "pggc_local_move": (_ci, [_vp, _vp, _vp, _vp, _ci, _ci, _vp, _i64, _ci, _ci, _ci, _ci, ctypes.POINTER(Stats)]),
    "pggc_select_pass": (_ci, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _flt, _ci, _ci, _vp, _ci, ctypes.POINTER(_i64)]),
    "pggc_build_coarse_graph": (_ci, [_vp, _vp, _vp, _i64, _ci, _PP]),
    "pggc_coarsen_leidenR": (_ci, [_vp, _vp, _vp, _vp, _u32, _u32, _vp, ctypes.POINTER(_i64), _ci]),
    "pggc_leiden_part": (_ci, [_vp, _vp, _vp, _ci, _ci, _vp, _u64, _vp, _ci, ctypes.POINTER(Stats)]),
    "pggc_louvain_part": (_ci, [_vp, _vp, _vp, _ci, _vp, _vp, _ci, ctypes.POINTER(Stats)]),
    "pggc_run_clustering": (_ci, [_vp, _vp, _vp, _ci, _ci, _u64, _vp, _ci, ctypes.POINTER(Stats)]),
    "pggc_verify_objective": (_ci, [_vp, _vp, _vp, _ci, _dbl, _ci, ctypes.POINTER(_dbl), ctypes.POINTER(_dbl)]),
}

EXPORTED = tuple(_SIGS)

_LIB = None


def lib():
    """Load (building first if absent) and return the CUDA library."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            _build.build_cuda()
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(status: int) -> None:
    if status == PGGC_OK:
        return
    msg = lib().pggc_last_error().decode(errors="replace")
    if status == PGGC_ERR_INVALID:
        raise InvalidArgument(status, msg)
    if status == PGGC_ERR_DEVICE:
        raise DeviceError(status, msg)
    raise PggcError(status, msg)
