"""Small graphs shared by the tests (hand-checkable shapes + seeded generators)."""
import numpy as np

from pennsylvaniagpugraphclustering_b200 import graphgen as gg
from pennsylvaniagpugraphclustering_b200.graphgen import HostGraph


def from_edges(n, edges, weights=None):
    """Symmetric CSR from an undirected edge list (no loops, no duplicates)."""
    src, dst, ww = [], [], []
    for k, (u, v) in enumerate(edges):
        src += [u, v]
        dst += [v, u]
        if weights is not None:
            ww += [weights[k], weights[k]]
    src = np.array(src, np.int64)
    dst = np.array(dst, np.int64)
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    rowptr = np.zeros(n + 1, np.int64)
    np.add.at(rowptr, src + 1, 1)
    rowptr = np.cumsum(rowptr)
    w = None
    if weights is not None:
        w = np.array(ww, np.float32)[order]
    return HostGraph(rowptr, dst.astype(np.int32), w, name="edges")


def two_cliques(k=6):
    edges = [(i, j) for i in range(k) for j in range(i + 1, k)]
    edges += [(k + i, k + j) for i in range(k) for j in range(i + 1, k)]
    edges.append((0, k))
    return from_edges(2 * k, edges)


def ring_of_cliques(nc=8, k=5):
    edges = []
    for c in range(nc):
        b = c * k
        edges += [(b + i, b + j) for i in range(k) for j in range(i + 1, k)]
        edges.append((b, ((c + 1) % nc) * k + 1))
    return from_edges(nc * k, edges)


def star(leaves=40):
    return from_edges(leaves + 1, [(0, i) for i in range(1, leaves + 1)])


def path(n=30):
    return from_edges(n, [(i, i + 1) for i in range(n - 1)])


def with_isolated(n_iso=7):
    g = two_cliques(5)
    n = g.n + n_iso
    rowptr = np.concatenate([g.rowptr, np.full(n_iso, g.rowptr[-1], np.int64)])
    return HostGraph(rowptr, g.col, None, name="two_cliques+isolated")


def hub_graph(hub_deg=16000, seed=3):
    """A graph with one massive (degree >= 15000) vertex plus SBM structure."""
    base = gg.sbm(hub_deg + 1, 16, 10.0, 2.0, seed)
    n = base.n
    rng = np.random.default_rng(seed)
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(base.rowptr))
    dst = base.col.astype(np.int64)
    mask = (src != 0) & (dst != 0)
    src, dst = src[mask], dst[mask]
    spokes = np.arange(1, n, dtype=np.int64)
    src = np.concatenate([src, np.zeros(n - 1, np.int64), spokes])
    dst = np.concatenate([dst, spokes, np.zeros(n - 1, np.int64)])
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    keep = np.ones(src.shape[0], bool)
    keep[1:] = (src[1:] != src[:-1]) | (dst[1:] != dst[:-1])
    src, dst = src[keep], dst[keep]
    rowptr = np.zeros(n + 1, np.int64)
    np.add.at(rowptr, src + 1, 1)
    rowptr = np.cumsum(rowptr)
    w = (0.5 + rng.random(dst.shape[0])).astype(np.float32)
    # symmetric weights: use the pair hash
    lo, hi = np.minimum(src, dst), np.maximum(src, dst)
    w = (0.5 + ((lo * 1000003 + hi * 7919) % 1000) / 1000.0).astype(np.float32)
    return HostGraph(rowptr, dst.astype(np.int32), w, name="hub")


def small_sbm(seed=1):
    return gg.sbm(4096, 16, 12.0, 3.0, seed)


def small_dcsbm(seed=1, n=20000):
    return gg.dcsbm(n, seed)


def small_rmat(seed=1, scale=12):
    return gg.rmat(scale, 16, 0.57, 0.19, 0.19, seed)


def int_weighted(hg, scale=4.0):
    """The same graph with int32 edge weights round(scale * w) (symmetric
    because w is): the reference's own weight type."""
    w = np.maximum(np.rint(hg.w.astype(np.float64) * scale), 1).astype(np.int32)
    return HostGraph(hg.rowptr, hg.col, w, name=hg.name + "+int")


def with_vertex_weights(hg, seed):
    """The same graph carrying custom vertex weights ``vw`` (int64 for uniform or
    int32-weighted graphs, float64 for FP32-weighted ones)."""
    rng = np.random.default_rng(seed)
    g = HostGraph(hg.rowptr, hg.col, hg.w, name=hg.name + "+vw")
    if hg.w is not None and hg.w.dtype == np.float32:
        # FP32 values: their FP64 sums are exact in any order, the condition
        # for bit-reproducible cluster volumes
        g.vw = rng.uniform(0.5, 3.0, hg.n).astype(np.float32).astype(np.float64)
    else:
        g.vw = rng.integers(1, 21, hg.n).astype(np.int64)
    return g


def symmetric_weights(hg):
    """FP32 weights in [0.5, 1.5) from a hash of the unordered pair (equal in
    both directions)."""
    src = np.repeat(np.arange(hg.n, dtype=np.int64), np.diff(hg.rowptr))
    dst = hg.col.astype(np.int64)
    lo, hi = np.minimum(src, dst), np.maximum(src, dst)
    return (0.5 + ((lo * 1000003 + hi * 7919) % 1000) / 1000.0).astype(np.float32)


def wide_int_weights(hg, hi=10000, seed=5):
    """The same graph with symmetric int32 weights in [1, hi] from a hash of the
    unordered pair: DeltaQ ties between clusters become vanishingly rare, so
    tie-breaking rules stop mattering.  Totals stay far below 2^31 for the
    test graphs (the reference sums weights in int32)."""
    src = np.repeat(np.arange(hg.n, dtype=np.int64), np.diff(hg.rowptr))
    dst = hg.col.astype(np.int64)
    lo, hh = np.minimum(src, dst), np.maximum(src, dst)
    h = (lo * 2654435761 + hh * 40503 + seed * 97) % 1000003
    w = (1 + (h * 7919) % hi).astype(np.int32)
    return HostGraph(hg.rowptr, hg.col, w, name=hg.name + "+wide")
