"""ctypes bindings of the reference's own clustering code (TEST INFRASTRUCTURE ONLY).

``oracle/_ref/libpggc_ref.so`` is the reference's src/*.cpp compiled
unmodified against serial stand-ins for Kokkos, KokkosKernels and thrust
(``oracle/ref_shim/``), with the C entry points of ``oracle/ref_harness.cpp``.
It exists only where the reference sources were present at build time
(``make -C oracle ref``); :func:`available` says whether it can be loaded.
Only tests/ import this module.

The reference's types are int32 vertex ids, int32 edge offsets and int32
weights (interface/core_types.h:8-14): graphs passed here have integer or unit
weights and fewer than 2^31 edges.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libpggc_ref.so")

_LIB = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _LIB
    if _LIB is None:
        L = ctypes.CDLL(LIB_PATH)
        vp, i64, ci, dbl, u64 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_double, ctypes.c_uint64
        P64, PD = ctypes.POINTER(i64), ctypes.POINTER(dbl)
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_generate_orderings.argtypes = [i64, i64, vp, vp, vp, vp, vp]
        L.ref_build_coarse_graph.argtypes = [i64, i64, vp, vp, vp, vp, i64, vp, vp, vp, i64, vp, P64]
        L.ref_local_move_initial.argtypes = [i64, i64, vp, vp, vp, ci, vp, PD, P64]
        L.ref_run_clustering.argtypes = [i64, i64, vp, vp, vp, vp, ci, dbl, ci, ci, u64, ci, vp, PD, P64, P64]
        L.ref_local_move_sweeps.argtypes = [i64, i64, vp, vp, vp, ci, ci, ci, ci, vp, PD, P64, P64]
        L.ref_local_move_then_refine.argtypes = [i64, i64, vp, vp, vp, ci, ctypes.c_uint32, ctypes.c_uint32, vp, vp,
                                                 P64]
        for f in (L.ref_generate_orderings, L.ref_build_coarse_graph, L.ref_local_move_initial, L.ref_run_clustering,
                  L.ref_local_move_sweeps, L.ref_local_move_then_refine):
            f.restype = ci
        _LIB = L
    return _LIB


def _check(status):
    if status != 0:
        raise RuntimeError(lib().ref_last_error().decode(errors="replace"))


def _csr(rowptr, col, w):
    rp = np.ascontiguousarray(rowptr, np.int64)
    c = np.ascontiguousarray(col, np.int32)
    ww = None if w is None else np.ascontiguousarray(w, np.int32)
    return rp, c, ww


def _p(a):
    return None if a is None else a.ctypes.data


def generate_orderings(rowptr, col):
    """ordering::generate_orderings -> (order1, order2, offsets[4])."""
    rp, c, _ = _csr(rowptr, col, None)
    n = len(rp) - 1
    o1, o2 = np.empty(max(n, 1), np.int32), np.empty(max(n, 1), np.int32)
    off = np.zeros(4, np.int64)
    _check(lib().ref_generate_orderings(n, len(c), _p(rp), _p(c), _p(o1), _p(o2), _p(off)))
    return o1[:n], o2[:n], off


def build_coarse_graph(rowptr, col, w, vcmap, nc):
    """contracter::build_coarse_graph -> (rowptr, col, w, vertex weights) of the
    coarse graph, rows in the reference's (hash-slot) order."""
    rp, c, ww = _csr(rowptr, col, w)
    n = len(rp) - 1
    m = np.ascontiguousarray(vcmap, np.int32)
    cap = max(len(c), 1)
    rpo = np.zeros(nc + 1, np.int64)
    co, wo = np.empty(cap, np.int32), np.empty(cap, np.int32)
    vwo = np.zeros(max(nc, 1), np.int64)
    nnz = ctypes.c_int64()
    _check(lib().ref_build_coarse_graph(n, len(c), _p(rp), _p(c), _p(ww), _p(m), nc, _p(rpo), _p(co), _p(wo), cap,
                                        _p(vwo), ctypes.byref(nnz)))
    k = nnz.value
    return rpo, co[:k], wo[:k], vwo[:nc]


def local_move_initial(rowptr, col, w, objective):
    """local_move<false> from singletons -> (labels, objective, label count)."""
    rp, c, ww = _csr(rowptr, col, w)
    n = len(rp) - 1
    lab = np.empty(max(n, 1), np.int32)
    q, L = ctypes.c_double(), ctypes.c_int64()
    _check(lib().ref_local_move_initial(n, len(c), _p(rp), _p(c), _p(ww), objective, _p(lab), ctypes.byref(q),
                                        ctypes.byref(L)))
    return lab[:n], q.value, L.value


def local_move_sweeps(rowptr, col, w, objective, part=None, enable_sa=True, sweep_limit=-1):
    """The reference's local_move<false> sweep loop stopped after sweep_limit
    sweeps, from singletons (part None) or from `part` -> (best labels,
    raw objective, label count, sweeps run)."""
    rp, c, ww = _csr(rowptr, col, w)
    n = len(rp) - 1
    initial = part is None
    lab = np.arange(max(n, 1), dtype=np.int32) if initial else np.ascontiguousarray(part, np.int32).copy()
    q, L, S = ctypes.c_double(), ctypes.c_int64(), ctypes.c_int64()
    _check(lib().ref_local_move_sweeps(n, len(c), _p(rp), _p(c), _p(ww), objective, int(initial), int(enable_sa),
                                       sweep_limit, _p(lab), ctypes.byref(q), ctypes.byref(L), ctypes.byref(S)))
    return lab[:n], q.value, L.value, S.value


def local_move_then_refine(rowptr, col, w, objective, seed_pick, seed_order):
    """The first level of leiden_part: initial local move, then
    coarsen_leidenR<top> of its partition with the given seeds ->
    (local-move labels, refinement map, coarse vertex count)."""
    rp, c, ww = _csr(rowptr, col, w)
    n = len(rp) - 1
    part, vcmap = np.empty(max(n, 1), np.int32), np.empty(max(n, 1), np.int32)
    nc = ctypes.c_int64()
    _check(lib().ref_local_move_then_refine(n, len(c), _p(rp), _p(c), _p(ww), objective, seed_pick & 0xFFFFFFFF,
                                            seed_order & 0xFFFFFFFF, _p(part), _p(vcmap), ctypes.byref(nc)))
    return part[:n], vcmap[:n], nc.value


def run_clustering(rowptr, col, w, objective, method, ex_iters=0, seed=1, vtx_w=None, lambda_mult=1.0,
                   sorted_rows=False):
    """run_clustering -> (labels, objective, label count, passes).  sorted_rows:
    pLeiden / pLeiden+ with every coarse graph's rows sorted by column (the
    CUDA library's and the oracle's row order) instead of hash-slot order."""
    rp, c, ww = _csr(rowptr, col, w)
    n = len(rp) - 1
    vw = None if vtx_w is None else np.ascontiguousarray(vtx_w, np.int64)
    lab = np.empty(max(n, 1), np.int32)
    q, L, P = ctypes.c_double(), ctypes.c_int64(), ctypes.c_int64()
    _check(lib().ref_run_clustering(n, len(c), _p(rp), _p(c), _p(ww), _p(vw), objective, float(lambda_mult), method,
                                    ex_iters, seed, int(sorted_rows), _p(lab), ctypes.byref(q), ctypes.byref(L),
                                    ctypes.byref(P)))
    return lab[:n], q.value, L.value, P.value
