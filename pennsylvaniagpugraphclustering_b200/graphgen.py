"""Seeded synthetic graphs standing in for the reference's external graph set.

Thin ctypes wrapper over ``csrc/graphgen.cpp``.  Every generator returns a
:class:`HostGraph`: a symmetric CSR (int64 row offsets, int32 columns sorted
within rows, no self-loops, no duplicates) with optional FP32 edge weights.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import build as _build

_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_build.OUT, "libpggc_graphgen.so")
        if not os.path.exists(path):
            path = _build.build_graphgen()
        lib = ctypes.CDLL(path)
        vp, i64, dbl, u64, flt, ci = (ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_uint64,
                                     ctypes.c_float, ctypes.c_int)
        lib.pggc_gen_sbm.argtypes = [i64, i64, dbl, dbl, u64, ci, flt, flt]
        lib.pggc_gen_sbm.restype = vp
        lib.pggc_gen_dcsbm.argtypes = [i64, dbl, dbl, dbl, dbl, dbl, i64, i64, dbl, u64, ci, flt, flt]
        lib.pggc_gen_dcsbm.restype = vp
        lib.pggc_gen_rmat.argtypes = [i64, i64, dbl, dbl, dbl, u64, ci, flt, flt]
        lib.pggc_gen_rmat.restype = vp
        lib.pggc_gen_dims.argtypes = [vp, ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(ci)]
        lib.pggc_gen_read.argtypes = [vp, vp, vp, vp]
        lib.pggc_gen_free.argtypes = [vp]
        lib.pggc_gen_free.restype = vp
        _LIB = lib
    return _LIB


@dataclass
class HostGraph:
    """Symmetric CSR in host memory."""
    rowptr: np.ndarray            # int64 [n+1]
    col: np.ndarray               # int32 [nnz]
    w: Optional[np.ndarray] = None  # float32 [nnz] or None (unit weights)
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.rowptr.shape[0] - 1)

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])

    @property
    def m(self) -> int:
        """Undirected edge count."""
        return self.nnz // 2


def _take(h) -> HostGraph:
    lib = _lib()
    n, nnz, hw = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int()
    lib.pggc_gen_dims(h, ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(hw))
    rowptr = np.empty(n.value + 1, dtype=np.int64)
    col = np.empty(nnz.value, dtype=np.int32)
    w = np.empty(nnz.value, dtype=np.float32) if hw.value else None
    lib.pggc_gen_read(h, rowptr.ctypes.data, col.ctypes.data, w.ctypes.data if w is not None else None)
    lib.pggc_gen_free(h)
    return HostGraph(rowptr, col, w)


def sbm(n: int, blocks: int, deg_in: float, deg_out: float, seed: int, weighted: bool = False,
        wlo: float = 0.5, whi: float = 1.5) -> HostGraph:
    """Planted-partition SBM; vertex v belongs to block v // (n // blocks)."""
    g = _take(_lib().pggc_gen_sbm(n, blocks, deg_in, deg_out, seed, int(weighted), wlo, whi))
    g.name = f"sbm(n={n},blocks={blocks},din={deg_in},dout={deg_out},seed={seed})"
    return g


def dcsbm(n: int, seed: int, deg_exp: float = 2.5, min_deg: float = 5.0, mean_deg: float = 20.0,
          max_deg: float = 2000.0, comm_exp: float = 1.5, cmin: int = 50, cmax: int = 5000, mu: float = 0.4,
          weighted: bool = True, wlo: float = 0.5, whi: float = 1.5) -> HostGraph:
    """Degree-corrected SBM with power-law degrees and community sizes."""
    g = _take(_lib().pggc_gen_dcsbm(n, deg_exp, min_deg, mean_deg, max_deg, comm_exp, cmin, cmax, mu, seed,
                                    int(weighted), wlo, whi))
    g.name = f"dcsbm(n={n},mu={mu},seed={seed},weighted={weighted})"
    return g


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 1,
         weighted: bool = False) -> HostGraph:
    """R-MAT, symmetrised, deduplicated, self-loops removed."""
    g = _take(_lib().pggc_gen_rmat(scale, edge_factor, a, b, c, seed, int(weighted), 0.5, 1.5))
    g.name = f"rmat(scale={scale},ef={edge_factor},seed={seed})"
    return g


# ---- the named workloads ---------------------------------------------------
def planted_sbm_65k(seed: int = 1) -> HostGraph:
    """pLouvain workload: n=65,536, 64 blocks of 1,024, expected degrees 16 / 4, unit weights."""
    return sbm(65536, 64, 16.0, 4.0, seed)


# Expected degree before deduplication that leaves a mean degree of 20 after
# it on the 4,194,304-vertex DC-SBM: pairs drawn twice inside small
# communities merge, so mean 20 would give 39.06 M edges instead of 41.9 M
# (seed 1: 41,931,980 undirected edges, mean degree 19.995).
DCSBM_4M_MEAN_DEG = 21.53


def dcsbm_4m(seed: int = 1, n: int = 4194304) -> HostGraph:
    """pLeiden+ workload: DC-SBM n=4,194,304, degree exp 2.5 (min 5, mean 20 after deduplication,
    ~41.9 M undirected edges), community exp 1.5 on [50, 5000], mu=0.4, FP32 weights uniform in
    [0.5, 1.5)."""
    return dcsbm(n, seed, mean_deg=DCSBM_4M_MEAN_DEG)


def rmat24(seed: int = 1, scale: int = 24) -> HostGraph:
    """Contraction stress workload: R-MAT scale 24, edge factor 16, a=0.57, b=c=0.19."""
    return rmat(scale, 16, 0.57, 0.19, 0.19, seed)


def sbm_population_params(count: int = 256, seed: int = 1, n_lo: int = 1000, n_hi: int = 200000,
                          b_lo: int = 8, b_hi: int = 512):
    """Sizes of the batched workload's uneven-size SBM population: vertex
    counts log-uniform in [n_lo, n_hi], block counts log-uniform in
    [b_lo, b_hi] (at most n // 16 so that every block holds at least 16
    vertices, enough for expected intra-block degree 12), and one generator
    seed per graph.  Returns a list of (n, blocks, seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi)))))
        b = int(round(np.exp(rng.uniform(np.log(b_lo), np.log(b_hi)))))
        b = max(1, min(b, n // 16))
        out.append((n, b, int(rng.integers(1, 1 << 31))))
    return out


def sbm_population(count: int = 256, seed: int = 1, deg_in: float = 12.0, deg_out: float = 3.0):
    """The batched workload's population: `count` independent planted-partition
    SBMs (unit weights, expected intra / inter degree 12 / 3) with the sizes of
    :func:`sbm_population_params`."""
    return [sbm(n, b, deg_in, deg_out, s) for n, b, s in sbm_population_params(count, seed)]
