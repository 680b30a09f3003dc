"""Host-side mirror of the reference's clustering interface.

Names follow the reference's public API (``interface/``):

* :class:`memory_store`  -- interface/memory_store.hpp:12-91 (a CUDA context:
  stream + device memory pool);
* :class:`weighted_graph` -- interface/weighted_graph.h:10-19;
* :class:`cluster_data` and the objective subclasses ``modularity``,
  ``constant_potts``, ``normalized_lcc`` -- interface/cluster_data.hpp:9-181,
  built by :func:`get_objective` (app/objective_helpers.hpp:9-22);
* :mod:`clustering_methods` functions ``leiden_part`` / ``louvain_part``
  (interface/clustering_methods.h:20-24) and the kernel-level entry points
  ``generate_orderings``, ``local_move``, ``local_move_strict``,
  ``build_coarse_graph``, ``coarsen_leidenR``.

Arrays may be numpy arrays (host memory; copied in/out by the call) or CUDA
torch tensors (device memory; used in place).  Every call goes through the C
ABI of ``libpggc_b200.so``; there is no CPU path.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

from . import _lib as L
from ._lib import (MEM_DEVICE, MEM_HOST, METHOD_LEIDEN, METHOD_LEIDEN_PLUS, METHOD_LOUVAIN, OBJ_CPM, OBJ_LCC,
                   OBJ_MOD, OBJ_NLCC, OBJ_WMOD, W_FLOAT32, W_INT32, W_UNIFORM, Stats, check)

NULL_PART, NO_MOVE, NEW_PART = -1, -3, -4
OBJECTIVES = {"Mod": OBJ_MOD, "WMod": OBJ_WMOD, "CPM": OBJ_CPM, "NLCC": OBJ_NLCC, "LCC": OBJ_LCC}


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(x, dtype, n=None, writable=False):
    """(pointer, mem_kind, keepalive) for a numpy array or torch tensor."""
    if x is None:
        return None, MEM_HOST, None
    if _is_torch(x):
        import torch
        tdt = {np.int32: torch.int32, np.int64: torch.int64, np.float32: torch.float32,
               np.float64: torch.float64, np.uint8: torch.uint8}[dtype]
        if x.dtype != tdt:
            raise TypeError(f"expected {tdt}, got {x.dtype}")
        if not x.is_contiguous():
            raise ValueError("tensor must be contiguous")
        if n is not None and x.numel() < n:
            raise ValueError(f"tensor has {x.numel()} elements, need {n}")
        return x.data_ptr(), (MEM_DEVICE if x.is_cuda else MEM_HOST), x
    a = np.asarray(x)
    if a.dtype != dtype:
        if writable:
            raise TypeError(f"expected {np.dtype(dtype)}, got {a.dtype}")
        a = a.astype(dtype)
    if not a.flags.c_contiguous:
        if writable:
            raise ValueError("array must be C-contiguous")
        a = np.ascontiguousarray(a)
    if n is not None and a.size < n:
        raise ValueError(f"array has {a.size} elements, need {n}")
    return a.ctypes.data, MEM_HOST, a


def _one_kind(*kinds):
    ks = {k for k in kinds if k is not None}
    if len(ks) > 1:
        raise ValueError("mixing host and device arrays in one call is not supported")
    return ks.pop() if ks else MEM_HOST


class memory_store:
    """A device context: one CUDA stream and the device memory pool.

    Mirrors interface/memory_store.hpp:12-91; graphs and cluster data created on
    a context must be released before it.
    """

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        check(L.lib().pggc_context_create(device, ctypes.byref(h)))
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    def stream(self) -> int:
        s = ctypes.c_void_p()
        check(L.lib().pggc_context_stream(self._h, ctypes.byref(s)))
        return int(s.value or 0)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().pggc_context_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class weighted_graph:
    """Device-resident symmetric CSR + vertex weights (interface/weighted_graph.h:10-19).

    ``edge_uniform`` graphs carry no weight array; ``vtx_w`` defaults to the
    objective's rule (app/io/vertex_weighting.cpp:27-42).
    """

    def __init__(self, mem: memory_store, rowptr, col, weights=None, objective: int = OBJ_MOD, vtx_w=None,
                 edge_uniform: Optional[bool] = None, _handle=None):
        self.mem = mem
        self.objective = objective
        if _handle is not None:
            self._h = _handle
        else:
            n = int(rowptr.shape[0]) - 1
            nnz = int(col.shape[0])
            if edge_uniform is None:
                # Mod and CPM treat edges as unit weight (app/objective_helpers.hpp:24-29)
                edge_uniform = weights is None or objective in (OBJ_MOD, OBJ_CPM)
            if edge_uniform:
                kind, wdt = W_UNIFORM, None
            else:
                is_float = str(weights.dtype).endswith("float32") or str(weights.dtype).endswith("float64")
                wdt = np.float32 if is_float else np.int32
                kind = W_FLOAT32 if is_float else W_INT32
            rp, k1, a1 = _ptr(rowptr, np.int64)
            cp, k2, a2 = _ptr(col, np.int32)
            wp, k3, a3 = (None, None, None) if kind == W_UNIFORM else _ptr(weights, wdt)
            vdt = np.float64 if kind == W_FLOAT32 else np.int64
            vp, k4, a4 = (None, None, None) if vtx_w is None else _ptr(vtx_w, vdt)
            mk = _one_kind(k1, k2, k3, k4)
            h = ctypes.c_void_p()
            check(L.lib().pggc_graph_create(mem.handle, n, nnz, rp, cp, wp, kind, vp, objective, mk, ctypes.byref(h)))
            self._h = h
        n, nnz, k = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int()
        check(L.lib().pggc_graph_dims(self._h, ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(k)))
        self.n, self.nnz, self.weight_kind = n.value, nnz.value, k.value

    @property
    def handle(self):
        return self._h

    @property
    def edge_uniform(self) -> bool:
        return self.weight_kind == W_UNIFORM

    @property
    def vdtype(self):
        return np.float64 if self.weight_kind == W_FLOAT32 else np.int64

    def to_host(self):
        """(rowptr, col, weights or None, vtx_w) as numpy arrays."""
        rowptr = np.empty(self.n + 1, np.int64)
        col = np.empty(self.nnz, np.int32)
        w = None
        if self.weight_kind != W_UNIFORM:
            w = np.empty(self.nnz, np.float32 if self.weight_kind == W_FLOAT32 else np.int32)
        vw = np.empty(self.n, self.vdtype)
        check(L.lib().pggc_graph_read(self.mem.handle, self._h, rowptr.ctypes.data, col.ctypes.data,
                                      None if w is None else w.ctypes.data, vw.ctypes.data, MEM_HOST))
        return rowptr, col, w, vw

    def set_vertex_weights(self, vtx_w):
        """Replaces the vertex weights (``n`` values; int64, or float64 for FP32-weighted graphs)."""
        if int(vtx_w.shape[0]) != self.n:
            raise ValueError(f"vtx_w has {int(vtx_w.shape[0])} values, the graph {self.n} vertices")
        vp, k, a = _ptr(vtx_w, self.vdtype)
        check(L.lib().pggc_graph_set_vertex_weights(self.mem.handle, self._h, vp, k))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().pggc_graph_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load_graph(mem: memory_store, path, objective: int = OBJ_MOD, vtx_w=None) -> weighted_graph:
    """Reads a Matrix Market (``.mtx``) or METIS file into a device graph
    (load_graph, app/io/io_mtx.cpp:336-345; load_mtx_graph :204-333;
    load_metis_graph, app/io/io_metis.cpp:64-181).

    Mod and CPM ignore file weights; ``wg.edge_uniform`` is the reference's
    ``uniform_ew`` after loading.  ``vtx_w`` (n values, e.g. from
    :func:`load_view`) replaces the objective's default vertex weights, as
    ``-vw_file`` does (app/io/vertex_weighting.cpp:27-30).  Malformed files
    raise ``PggcError``.
    """
    h = ctypes.c_void_p()
    uni = ctypes.c_int()
    check(L.lib().pggc_graph_load(mem.handle, os.fsencode(str(path)), objective, ctypes.byref(uni), ctypes.byref(h)))
    wg = weighted_graph(mem, None, None, objective=objective, _handle=h)
    if vtx_w is not None:
        wg.set_vertex_weights(vtx_w)
    return wg


def load_view(n: int, path, dtype=np.int64) -> np.ndarray:
    """``load_view<view_t>(n, fname)`` (app/io/header/io_views.hpp:26-41): the
    first ``n`` whitespace-separated values of a text file (vertex weights for
    ``-vw_file``, a clustering for verify_objective).  A file that cannot be
    opened raises ``InvalidArgument`` (the reference prints FATAL ERROR and
    returns zeros); values the file does not hold stay 0, as in the reference."""
    try:
        with open(path, "rb") as fh:
            tokens = fh.read().split()
    except OSError as e:
        raise L.InvalidArgument(L.PGGC_ERR_INVALID, f"could not open {path}: {e}") from None
    out = np.zeros(int(n), dtype)
    k = min(int(n), len(tokens))
    if k:
        out[:k] = np.array(tokens[:k]).astype(dtype)
    return out


def write_part(labels, path) -> None:
    """``write_part`` (app/io/header/io_views.hpp:11-24): one label per line."""
    a = np.asarray(labels.cpu() if hasattr(labels, "cpu") else labels).ravel()
    with open(path, "w") as fh:
        fh.write("".join(f"{int(x)}\n" for x in a))

def graph_from_edges(mem: memory_store, n: int, src, dst, weights=None, symmetric: bool = True,
                     objective: int = OBJ_MOD) -> weighted_graph:
    """Builds the CSR of a 0-based edge list on the GPU (construct_from_edgelist,
    app/io/io_mtx.cpp:95-201): self loops and zero-weight entries dropped,
    both directions stored, unordered duplicates removed unless ``symmetric``,
    rows sorted by column.  ``weights`` (int32) only for symmetric lists."""
    m = int(src.shape[0])
    if int(dst.shape[0]) != m or (weights is not None and int(weights.shape[0]) != m):
        raise ValueError("src, dst and weights must have the same length")
    sp, k1, a1 = _ptr(src, np.int32)
    dp, k2, a2 = _ptr(dst, np.int32)
    wp, k3, a3 = (None, None, None) if weights is None else _ptr(weights, np.int32)
    mk = _one_kind(k1, k2, k3)
    h = ctypes.c_void_p()
    check(L.lib().pggc_graph_from_edges(mem.handle, int(n), m, sp, dp, wp, int(bool(symmetric)), objective, mk,
                                        ctypes.byref(h)))
    return weighted_graph(mem, None, None, objective=objective, _handle=h)


class cluster_data:
    """Objective state (interface/cluster_data.hpp:9-107): total_deg, uncut,
    obj, label_count, lambda.  Subclasses fix lambda and the normalisation."""

    objective_kind = OBJ_LCC

    def __init__(self, mem: memory_store, g: weighted_graph, lambda_mult: float = 1.0, objective=None):
        self.mem = mem
        self.graph = g
        kind = self.objective_kind if objective is None else objective
        h = ctypes.c_void_p()
        check(L.lib().pggc_cluster_data_create(mem.handle, g.handle, kind, lambda_mult, ctypes.byref(h)))
        self._h = h
        self.kind = kind

    @property
    def handle(self):
        return self._h

    def _get(self):
        o, ob, lam, un = (ctypes.c_double() for _ in range(4))
        lc = ctypes.c_int64()
        check(L.lib().pggc_cluster_data_get(self._h, ctypes.byref(o), ctypes.byref(ob), ctypes.byref(lam),
                                            ctypes.byref(un), ctypes.byref(lc)))
        return o.value, ob.value, lam.value, un.value, lc.value

    @property
    def obj(self) -> float:
        return self._get()[0]

    def get_objective(self) -> float:
        return self._get()[1]

    @property
    def lambda_(self) -> float:
        return self._get()[2]

    @property
    def uncut(self) -> float:
        return self._get()[3]

    @property
    def label_count(self) -> int:
        return self._get()[4]

    def total_deg(self):
        out = np.empty(self.label_count, self.graph.vdtype)
        check(L.lib().pggc_cluster_data_total_deg(self.mem.handle, self._h, out.ctypes.data, MEM_HOST))
        return out

    def set_state(self, label_count: int, total_deg, uncut: float):
        p, mk, keep = _ptr(total_deg, self.graph.vdtype)
        check(L.lib().pggc_cluster_data_set(self.mem.handle, self._h, label_count, p, float(uncut), mk))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().pggc_cluster_data_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class modularity(cluster_data):
    """lambda = mult / w(E); objective = obj / w(E) (interface/cluster_data.hpp:109-133)."""
    objective_kind = OBJ_MOD

    def __init__(self, mem, g, lambda_mult=1.0, uniform=True):
        super().__init__(mem, g, lambda_mult, OBJ_MOD if uniform or g.edge_uniform else OBJ_WMOD)


class constant_potts(cluster_data):
    """lambda = mult / 2; objective = obj + lambda * n (interface/cluster_data.hpp:135-156)."""
    objective_kind = OBJ_CPM


class normalized_lcc(cluster_data):
    """lambda = mult * w(E) / w(V)^2; objective = obj / w(E) (interface/cluster_data.hpp:158-181)."""
    objective_kind = OBJ_NLCC


def get_objective(mem: memory_store, g: weighted_graph, objective: int, lambda_mult: float = 1.0) -> cluster_data:
    """app/objective_helpers.hpp:9-22."""
    return cluster_data(mem, g, lambda_mult, objective)


def _stats_dict(st: Stats):
    return st.as_dict()


# ---- kernel-level entry points -------------------------------------------
def generate_orderings(mem: memory_store, g: weighted_graph):
    """src/ordering.cpp:131-164 -> (order1, order2, offsets[4]) as numpy arrays."""
    o1, o2 = np.empty(g.n, np.int32), np.empty(g.n, np.int32)
    off = np.zeros(4, np.int64)
    check(L.lib().pggc_generate_orderings(mem.handle, g.handle, o1.ctypes.data, o2.ctypes.data, off.ctypes.data,
                                          MEM_HOST))
    return o1, o2, off


def local_move(mem, g, part, rfd, is_initial, constraint=None, enable_simulated_annealing=True, sweep_limit=-1):
    """local_move<constrained> (src/local_mover.cpp:1361-1417); part and rfd are updated in place."""
    return _local_move(mem, g, part, rfd, is_initial, constraint, enable_simulated_annealing, False, sweep_limit)


def local_move_strict(mem, g, part, rfd, is_initial, constraint=None, sweep_limit=-1):
    """local_move_strict<constrained> (src/local_mover.cpp:1422-1483)."""
    return _local_move(mem, g, part, rfd, is_initial, constraint, False, True, sweep_limit)


def _local_move(mem, g, part, rfd, is_initial, constraint, sa, strict, sweep_limit):
    pp, k1, a1 = _ptr(part, np.int32, g.n, writable=True)
    cp, k2, a2 = _ptr(constraint, np.int32, writable=True) if constraint is not None else (None, None, None)
    mk = _one_kind(k1, k2)
    st = Stats()
    clen = 0 if constraint is None else int(constraint.shape[0])
    check(L.lib().pggc_local_move(mem.handle, g.handle, rfd.handle, pp, int(is_initial), int(constraint is not None),
                                  cp, clen, int(sa), int(strict), sweep_limit, mk, ctypes.byref(st)))
    return _stats_dict(st)


def select_pass(mem, g, rfd, part, pvals, dest, filter_ratio, initial, constraint=None, gain=None):
    """One candidates_and_destinations pass; returns (dest, gain, num_candidates).

    ``gain`` is save_gains in/out (zeros when omitted): vertices skipped by the
    dest cache keep their entries."""
    dest = np.array(dest, np.int32, copy=True)
    gain = np.zeros(g.n, np.float32) if gain is None else np.array(gain, np.float32, copy=True)
    pp, _, a1 = _ptr(part, np.int32)
    vp, _, a2 = _ptr(pvals, g.vdtype)
    cp, _, a3 = _ptr(constraint, np.int32) if constraint is not None else (None, None, None)
    k = ctypes.c_int64()
    check(L.lib().pggc_select_pass(mem.handle, g.handle, rfd.handle, pp, vp, dest.ctypes.data, gain.ctypes.data,
                                   float(filter_ratio), int(initial), int(constraint is not None), cp, MEM_HOST,
                                   ctypes.byref(k)))
    return dest, gain, k.value


def build_coarse_graph(mem, g, vcmap, nc) -> weighted_graph:
    """src/contract.cpp:234-336; returns the coarse weighted_graph (rows sorted)."""
    vp, mk, keep = _ptr(vcmap, np.int32, g.n)
    h = ctypes.c_void_p()
    check(L.lib().pggc_build_coarse_graph(mem.handle, g.handle, vp, int(nc), mk, ctypes.byref(h)))
    return weighted_graph(mem, None, None, _handle=h)


def coarsen_leidenR(mem, g, constraint, rfd, seed_pick: int, seed_order: int):
    """src/leidenR.cpp:263-500 -> (vcmap, coarse_vtx_count)."""
    cp, mk, keep = _ptr(constraint, np.int32, g.n)
    out = np.empty(g.n, np.int32)
    nc = ctypes.c_int64()
    if mk == MEM_DEVICE:
        import torch
        outt = torch.empty(g.n, dtype=torch.int32, device=constraint.device)
        check(L.lib().pggc_coarsen_leidenR(mem.handle, g.handle, rfd.handle, cp, seed_pick & 0xFFFFFFFF,
                                           seed_order & 0xFFFFFFFF, outt.data_ptr(), ctypes.byref(nc), MEM_DEVICE))
        return outt, nc.value
    check(L.lib().pggc_coarsen_leidenR(mem.handle, g.handle, rfd.handle, cp, seed_pick & 0xFFFFFFFF,
                                       seed_order & 0xFFFFFFFF, out.ctypes.data, ctypes.byref(nc), MEM_HOST))
    return out, nc.value


def verify_objective(mem, g, labels, objective=OBJ_MOD, lambda_mult=1.0):
    """app/verify_objective.cpp:64-89 -> (objective, raw obj)."""
    lp, mk, keep = _ptr(labels, np.int32, g.n)
    o, r = ctypes.c_double(), ctypes.c_double()
    check(L.lib().pggc_verify_objective(mem.handle, g.handle, lp, objective, lambda_mult, mk, ctypes.byref(o),
                                        ctypes.byref(r)))
    return o.value, r.value


def _labels_out(g, like):
    if like is not None and _is_torch(like) and like.is_cuda:
        import torch
        return torch.empty(g.n, dtype=torch.int32, device=like.device)
    return np.empty(g.n, np.int32)


class clustering_methods:
    """interface/clustering_methods.h:20-24; template flags become keywords."""

    @staticmethod
    def leiden_part(mem, top, rfd, input=None, plus=True, improve=False, seed=1, out=None):
        labels = out if out is not None else _labels_out(top, input)
        lp, k1, a1 = _ptr(labels, np.int32, top.n, writable=True)
        ip, k2, a2 = _ptr(input, np.int32, top.n) if input is not None else (None, None, None)
        mk = _one_kind(k1, k2)
        st = Stats()
        check(L.lib().pggc_leiden_part(mem.handle, top.handle, rfd.handle, int(plus), int(improve), ip, seed, lp, mk,
                                       ctypes.byref(st)))
        return labels, _stats_dict(st)

    @staticmethod
    def louvain_part(mem, top, rfd, constraint=None, out=None):
        labels = out if out is not None else _labels_out(top, constraint)
        lp, k1, a1 = _ptr(labels, np.int32, top.n, writable=True)
        cp, k2, a2 = _ptr(constraint, np.int32, top.n) if constraint is not None else (None, None, None)
        mk = _one_kind(k1, k2)
        st = Stats()
        check(L.lib().pggc_louvain_part(mem.handle, top.handle, rfd.handle, int(constraint is not None), cp, lp, mk,
                                        ctypes.byref(st)))
        return labels, _stats_dict(st)


def run_clustering(mem, g, rfd, method=METHOD_LEIDEN_PLUS, ex_iters=0, seed=1, out=None):
    """run_clustering (app/cluster_main.cpp:116-165) -> (labels, stats)."""
    labels = out if out is not None else np.empty(g.n, np.int32)
    lp, mk, keep = _ptr(labels, np.int32, g.n, writable=True)
    st = Stats()
    check(L.lib().pggc_run_clustering(mem.handle, g.handle, rfd.handle, method, ex_iters, seed, lp, mk,
                                      ctypes.byref(st)))
    return labels, _stats_dict(st)


def _batch_jobs(jobs):
    arr = (L.BatchJob * max(len(jobs), 1))()
    outs = []
    for k, j in enumerate(jobs):
        g = j["graph"]
        lab = np.empty(max(g.n, 1), np.int32)
        outs.append(lab)
        arr[k].graph = g.handle
        arr[k].objective = int(j.get("objective", g.objective))
        arr[k].lambda_mult = float(j.get("lambda_mult", 1.0))
        arr[k].method = int(j.get("method", METHOD_LEIDEN_PLUS))
        arr[k].ex_iters = int(j.get("ex_iters", 0))
        arr[k].seed = int(j.get("seed", 1))
        arr[k].labels_out = lab.ctypes.data
        arr[k].mem_kind = MEM_HOST
    return arr, outs


def batch_run(mem: memory_store, jobs, streams: int = 8):
    """Run independent clustering jobs concurrently (``pggc_batch_run``).

    ``jobs`` is a list of dicts with keys ``graph`` (a :class:`weighted_graph`
    of ``mem``), and optionally ``objective`` (default: the graph's),
    ``lambda_mult`` (1.0), ``method`` (pLeiden+), ``ex_iters`` (0) and
    ``seed`` (1).  ``streams`` = 0 uses the context's tuned batch width.
    Returns a list of (labels, stats dict) in job order.
    """
    arr, outs = _batch_jobs(jobs)
    check(L.lib().pggc_batch_run(mem.handle, ctypes.cast(arr, ctypes.c_void_p), len(jobs), int(streams)))
    return [(outs[k][:jobs[k]["graph"].n], _stats_dict(arr[k].stats)) for k in range(len(jobs))]


def tune_get(mem: memory_store) -> dict:
    """The context's kernel-selection knobs and batch width (``pggc_tune_get``)."""
    t = L.Tune()
    check(L.lib().pggc_tune_get(mem.handle, ctypes.byref(t)))
    return t.as_dict()


def tune_set(mem: memory_store, thread_max_deg=32, warp_max_deg=127, load_factor=0.5, streams=4) -> dict:
    """Set the knobs (``pggc_tune_set``; rounded to supported values); returns them."""
    t = L.Tune(int(thread_max_deg), int(warp_max_deg), float(load_factor), int(streams))
    check(L.lib().pggc_tune_set(mem.handle, ctypes.byref(t)))
    return tune_get(mem)


def batch_autotune(mem: memory_store, jobs):
    """Tune batch width, select degree bounds and table load factor on a sample
    batch (``pggc_batch_autotune``); the best setting stays on the context.
    Returns (best dict, [trial dicts])."""
    arr, _ = _batch_jobs(jobs)
    cap = 64
    trials = (L.TuneTrial * cap)()
    nt = ctypes.c_int64()
    best = L.Tune()
    check(L.lib().pggc_batch_autotune(mem.handle, ctypes.cast(arr, ctypes.c_void_p), len(jobs),
                                      ctypes.cast(trials, ctypes.c_void_p), cap, ctypes.byref(nt),
                                      ctypes.byref(best)))
    out = [dict(trials[k].config.as_dict(), seconds=trials[k].seconds, edges_per_s=trials[k].edges_per_s)
           for k in range(min(nt.value, cap))]
    return best.as_dict(), out


def meme_cluster(mem: memory_store, g: weighted_graph, objective=None, lambda_mult: float = 1.0, pop_size: int = 8,
                 offspring: int = 16, time_limit_s: float = 0.0, seed: int = 1):
    """Memetic clustering (app/memetic_clustering.cpp:118-219); returns (labels, stats dict)."""
    obj = g.objective if objective is None else objective
    lab = np.empty(max(g.n, 1), np.int32)
    st = L.MemeStats()
    check(L.lib().pggc_meme_cluster(mem.handle, g.handle, int(obj), float(lambda_mult), int(pop_size), int(offspring),
                                    float(time_limit_s), int(seed), lab.ctypes.data, MEM_HOST, ctypes.byref(st)))
    return lab[:g.n], st.as_dict()


def intersect_clusters(mem: memory_store, c1, c2):
    """intersection_cluster (app/memetic_clustering.cpp:27-62): (labels, count)."""
    a = np.ascontiguousarray(c1, np.int32)
    b = np.ascontiguousarray(c2, np.int32)
    out = np.empty(max(len(a), 1), np.int32)
    k = ctypes.c_int64()
    check(L.lib().pggc_intersect_clusters(mem.handle, a.ctypes.data, b.ctypes.data, len(a), out.ctypes.data,
                                          ctypes.byref(k), MEM_HOST))
    return out[:len(a)], k.value


def cut_signature(mem: memory_store, g: weighted_graph, labels):
    """gen_signature (app/memetic_clustering.cpp:64-104): uint32 words, bit j = edge j is cut."""
    lab = np.ascontiguousarray(labels, np.int32)
    out = np.empty(max((g.nnz + 31) // 32, 1), np.uint32)
    check(L.lib().pggc_cut_signature(mem.handle, g.handle, lab.ctypes.data, out.ctypes.data, MEM_HOST))
    return out
