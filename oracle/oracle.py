"""ctypes bindings of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference
leg may import this module; the product path never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libpggc_oracle.so")

W_UNIFORM, W_INT32, W_FLOAT32 = 0, 1, 2
OBJ_MOD, OBJ_WMOD, OBJ_CPM, OBJ_NLCC, OBJ_LCC = 0, 1, 2, 3, 4
METHOD_LOUVAIN, METHOD_LEIDEN, METHOD_LEIDEN_PLUS = 0, 1, 2

NULL_PART, NO_MOVE, NEW_PART = -1, -3, -4


class Stats(ctypes.Structure):
    _fields_ = [("levels", ctypes.c_int64), ("total_nnz", ctypes.c_int64), ("sweeps", ctypes.c_int64),
                ("moves", ctypes.c_int64), ("objective", ctypes.c_double), ("raw_obj", ctypes.c_double),
                ("label_count", ctypes.c_int64)]


_LIB = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, i64, ci, dbl, u32, u64, flt = (ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_uint32, ctypes.c_uint64, ctypes.c_float)
        L.orc_graph_new.argtypes = [i64, i64, vp, vp, vp, ci, vp, ci]
        L.orc_graph_new.restype = vp
        L.orc_graph_free.argtypes = [vp]
        L.orc_graph_dims.argtypes = [vp, ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(ci)]
        L.orc_graph_read.argtypes = [vp, vp, vp, vp, vp]
        L.orc_cd_new.argtypes = [vp, ci, dbl]
        L.orc_cd_new.restype = vp
        L.orc_cd_free.argtypes = [vp]
        L.orc_cd_get.argtypes = [vp, vp]
        L.orc_cd_total_deg.argtypes = [vp, vp]
        L.orc_cd_set.argtypes = [vp, i64, vp, dbl]
        L.orc_generate_orderings.argtypes = [i64, vp, vp, vp, vp]
        L.orc_build_coarse_graph.argtypes = [vp, vp, i64]
        L.orc_build_coarse_graph.restype = vp
        L.orc_select.argtypes = [vp, vp, vp, vp, vp, vp, flt, ci, ci, vp]
        L.orc_select.restype = i64
        L.orc_local_move.argtypes = [vp, vp, vp, ci, ci, vp, i64, ci, ci, ci, ctypes.POINTER(Stats)]
        L.orc_local_move.restype = ci
        L.orc_coarsen_leidenR.argtypes = [vp, vp, vp, u32, u32, vp]
        L.orc_coarsen_leidenR.restype = i64
        L.orc_run_clustering.argtypes = [vp, vp, ci, ci, u64, vp, ctypes.POINTER(Stats)]
        L.orc_leiden_part.argtypes = [vp, vp, ci, ci, vp, u64, vp, ctypes.POINTER(Stats)]
        L.orc_louvain_part.argtypes = [vp, vp, ci, vp, vp, ctypes.POINTER(Stats)]
        L.orc_verify_objective.argtypes = [vp, vp, ci, dbl, ctypes.POINTER(dbl)]
        L.orc_verify_objective.restype = dbl
        L.orc_connected_components.argtypes = [i64, vp, vp, vp]
        L.orc_connected_components.restype = i64
        L.orc_det_scan.argtypes = [vp, vp, i64]
        L.orc_det_reduce.argtypes = [vp, i64]
        L.orc_det_reduce.restype = dbl
        L.orc_murmur3.argtypes = [u32]
        L.orc_murmur3.restype = u32
        L.orc_num_threads.restype = ci
        L.orc_set_afterburner_reference_order.argtypes = [ci]
        L.orc_intersect.argtypes = [vp, vp, i64, vp]
        L.orc_intersect.restype = i64
        L.orc_signature.argtypes = [vp, vp, vp]
        L.orc_meme_cluster.argtypes = [vp, ci, dbl, ci, i64, u64, vp, ctypes.POINTER(MemeStats)]
        L.orc_meme_cluster.restype = ci
        L.orc_run_clustering.restype = ci
        L.orc_leiden_part.restype = ci
        L.orc_louvain_part.restype = ci
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_last_error.argtypes = []
        _LIB = L
    return _LIB


def set_afterburner_reference_order(on: bool) -> None:
    """Test switch: sum the afterburner's change and the strict prefix's gains
    in FP32 in the reference's order (on) instead of the canonical FP64
    association the CUDA library uses (off, the default) -- for step-by-step
    comparisons with the reference's own code (oracle/ref.py)."""
    lib().orc_set_afterburner_reference_order(1 if on else 0)


class MemeStats(ctypes.Structure):
    _fields_ = [("objective", ctypes.c_double), ("label_count", ctypes.c_int64), ("offspring", ctypes.c_int64),
                ("replaced", ctypes.c_int64), ("best_initial", ctypes.c_double)]


def _p(a):
    return None if a is None else a.ctypes.data


class Graph:
    """Oracle-side weighted_graph (copies the arrays)."""

    def __init__(self, rowptr, col, w=None, wkind=None, vtx_w=None, objective=OBJ_MOD, _handle=None):
        L = lib()
        if _handle is not None:
            self.h = _handle
        else:
            rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
            col = np.ascontiguousarray(col, dtype=np.int32)
            if wkind is None:
                wkind = W_UNIFORM if w is None else (W_FLOAT32 if w.dtype == np.float32 else W_INT32)
            if w is not None:
                w = np.ascontiguousarray(w, dtype=np.float32 if wkind == W_FLOAT32 else np.int32)
            if vtx_w is not None:
                vtx_w = np.ascontiguousarray(vtx_w, dtype=np.float64 if wkind == W_FLOAT32 else np.int64)
            self.h = L.orc_graph_new(rowptr.shape[0] - 1, col.shape[0], _p(rowptr), _p(col),
                                     _p(w) if wkind != W_UNIFORM else None, wkind, _p(vtx_w), objective)
        n, nnz, k = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int()
        L.orc_graph_dims(self.h, ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(k))
        self.n, self.nnz, self.wkind = n.value, nnz.value, k.value

    def __del__(self):
        if getattr(self, "h", None) and _LIB is not None:
            _LIB.orc_graph_free(self.h)
            self.h = None

    def arrays(self):
        rowptr = np.empty(self.n + 1, np.int64)
        col = np.empty(self.nnz, np.int32)
        w = None
        if self.wkind != W_UNIFORM:
            w = np.empty(self.nnz, np.float32 if self.wkind == W_FLOAT32 else np.int32)
        vw = np.empty(self.n, np.float64 if self.wkind == W_FLOAT32 else np.int64)
        lib().orc_graph_read(self.h, _p(rowptr), _p(col), _p(w), _p(vw))
        return rowptr, col, w, vw


class ClusterData:
    def __init__(self, graph: Graph, objective=OBJ_MOD, mult=1.0):
        self.graph = graph
        self.h = lib().orc_cd_new(graph.h, objective, mult)

    def __del__(self):
        if getattr(self, "h", None) and _LIB is not None:
            _LIB.orc_cd_free(self.h)
            self.h = None

    def info(self):
        out = np.empty(5, np.float64)
        lib().orc_cd_get(self.h, _p(out))
        return {"obj": out[0], "objective": out[1], "lambda": out[2], "uncut": out[3], "label_count": int(out[4])}

    def total_deg(self):
        L = self.info()["label_count"]
        out = np.empty(L, np.float64 if self.graph.wkind == W_FLOAT32 else np.int64)
        lib().orc_cd_total_deg(self.h, _p(out))
        return out

    def set_state(self, total_deg, uncut):
        td = np.ascontiguousarray(total_deg, dtype=np.float64 if self.graph.wkind == W_FLOAT32 else np.int64)
        lib().orc_cd_set(self.h, td.shape[0], _p(td), float(uncut))


def generate_orderings(rowptr):
    rowptr = np.ascontiguousarray(rowptr, np.int64)
    n = rowptr.shape[0] - 1
    o1, o2 = np.empty(n, np.int32), np.empty(n, np.int32)
    off = np.empty(4, np.int64)
    lib().orc_generate_orderings(n, _p(rowptr), _p(o1), _p(o2), _p(off))
    return o1, o2, off


def build_coarse_graph(g: Graph, vcmap, nc) -> Graph:
    vcmap = np.ascontiguousarray(vcmap, np.int32)
    h = lib().orc_build_coarse_graph(g.h, _p(vcmap), nc)
    return Graph(None, None, _handle=h)


def select(g: Graph, cd: ClusterData, part, pvals, dest, filter_ratio, initial, constrained=False, constraint=None,
           gain=None):
    part = np.ascontiguousarray(part, np.int32)
    pvals = np.ascontiguousarray(pvals, np.float64 if g.wkind == W_FLOAT32 else np.int64)
    dest = np.array(dest, np.int32, copy=True)
    gain = np.zeros(g.n, np.float32) if gain is None else np.array(gain, np.float32, copy=True)
    con = None if constraint is None else np.ascontiguousarray(constraint, np.int32)
    k = lib().orc_select(g.h, cd.h, _p(part), _p(pvals), _p(dest), _p(gain), filter_ratio, int(initial),
                         int(constrained), _p(con))
    return dest, gain, int(k)


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().orc_last_error().decode())


def local_move(g: Graph, cd: ClusterData, part, is_initial, enable_sa=True, strict=False, constrained=False,
               constraint=None, sweep_limit=-1):
    part = np.array(part, np.int32, copy=True)
    con = None if constraint is None else np.array(constraint, np.int32, copy=True)
    st = Stats()
    lib().orc_local_move(g.h, cd.h, _p(part), int(is_initial), int(constrained), _p(con),
                         0 if con is None else con.shape[0], int(enable_sa), int(strict), sweep_limit,
                         ctypes.byref(st))
    return part, st, con


def coarsen_leidenR(g: Graph, cd: ClusterData, constraint, seed_pick, seed_order):
    con = np.ascontiguousarray(constraint, np.int32)
    out = np.empty(g.n, np.int32)
    nc = lib().orc_coarsen_leidenR(g.h, cd.h, _p(con), seed_pick & 0xFFFFFFFF, seed_order & 0xFFFFFFFF, _p(out))
    return out, int(nc)


def run_clustering(g: Graph, cd: ClusterData, method=METHOD_LEIDEN_PLUS, ex_iters=0, seed=1):
    out = np.empty(g.n, np.int32)
    st = Stats()
    _check(lib().orc_run_clustering(g.h, cd.h, method, ex_iters, seed, _p(out), ctypes.byref(st)))
    return out, st


def leiden_part(g: Graph, cd: ClusterData, plus=True, improve=False, input_part=None, seed=1):
    out = np.empty(g.n, np.int32)
    st = Stats()
    inp = None if input_part is None else np.ascontiguousarray(input_part, np.int32)
    _check(lib().orc_leiden_part(g.h, cd.h, int(plus), int(improve), _p(inp), seed, _p(out), ctypes.byref(st)))
    return out, st


def louvain_part(g: Graph, cd: ClusterData, constrained=False, constraint=None):
    out = np.empty(g.n, np.int32)
    st = Stats()
    con = None if constraint is None else np.ascontiguousarray(constraint, np.int32)
    _check(lib().orc_louvain_part(g.h, cd.h, int(constrained), _p(con), _p(out), ctypes.byref(st)))
    return out, st


def verify_objective(g: Graph, labels, objective=OBJ_MOD, mult=1.0):
    labels = np.ascontiguousarray(labels, np.int32)
    raw = ctypes.c_double()
    val = lib().orc_verify_objective(g.h, _p(labels), objective, mult, ctypes.byref(raw))
    return val, raw.value


def connected_components(rowptr, col, labels) -> int:
    rowptr = np.ascontiguousarray(rowptr, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    labels = np.ascontiguousarray(labels, np.int32)
    return int(lib().orc_connected_components(rowptr.shape[0] - 1, _p(rowptr), _p(col), _p(labels)))


def det_scan(a):
    a = np.ascontiguousarray(a, np.float64)
    out = np.empty_like(a)
    lib().orc_det_scan(_p(a), _p(out), a.shape[0])
    return out


def det_reduce(a) -> float:
    a = np.ascontiguousarray(a, np.float64)
    return float(lib().orc_det_reduce(_p(a), a.shape[0]))


def murmur3(k: int) -> int:
    return int(lib().orc_murmur3(k & 0xFFFFFFFF))


# ---- memetic driver (app/memetic_clustering.cpp:27-219) -----------------------
def intersect(c1, c2):
    """intersection_cluster with canonical ids (ranks of the sorted distinct pairs)."""
    a = np.ascontiguousarray(c1, np.int32)
    b = np.ascontiguousarray(c2, np.int32)
    out = np.empty(len(a), np.int32)
    k = lib().orc_intersect(_p(a), _p(b), len(a), _p(out))
    return out, k


def signature(g: Graph, labels):
    lab = np.ascontiguousarray(labels, np.int32)
    out = np.empty(max((g.nnz + 31) // 32, 1), np.uint32)
    lib().orc_signature(g.h, _p(lab), _p(out))
    return out


def meme_cluster(g: Graph, objective, lambda_mult=1.0, pop_size=8, offspring=16, seed=1):
    out = np.empty(g.n, np.int32)
    st = MemeStats()
    _check(lib().orc_meme_cluster(g.h, objective, float(lambda_mult), pop_size, offspring, seed, _p(out), ctypes.byref(st)))
    return out, st
