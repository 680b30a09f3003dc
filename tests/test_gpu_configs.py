"""GPU parity on the named workload graphs at (or near) their full sizes.

* planted-partition SBM, n = 65,536 in 64 blocks of 1,024, expected degrees
  16 / 4, seed 1: modularity, pLouvain, one pass and until stable;
* degree-corrected SBM, n = 4,194,304 (the pLeiden+ benchmark graph), WMod,
  pLeiden+ first pass (ex_iters = 0);
* R-MAT scale 22 (edge factor 16, a = 0.57, b = c = 0.19), modularity,
  pLouvain, and its level-0 contraction: hub rows above 15,000 edges (the
  massive bucket, src/header/ordering.h:19) and a coarse graph of ~1.8 M
  vertices (large hash merges, placement above the shared-bitmap limit).

Every comparison is exact (labels, objective, label count, levels, coarse
CSR): the CUDA path and the oracle share one canonical arithmetic.
"""
import numpy as np
import pytest

import pennsylvaniagpugraphclustering_b200 as pg
from oracle import oracle as O
from pennsylvaniagpugraphclustering_b200 import graphgen as gg

pytestmark = pytest.mark.gpu

_G = {}


def graph(name):
    if name not in _G:
        if name == "sbm65k":
            _G[name] = gg.planted_sbm_65k(1)
        elif name == "dcsbm4m":
            _G[name] = gg.dcsbm_4m(1)
        elif name == "rmat22":
            _G[name] = gg.rmat(22, 16, 0.57, 0.19, 0.19, 1)
    return _G[name]


def _both(mem, hg, obj):
    w = hg.w if obj == pg.OBJ_WMOD else None
    og = O.Graph(hg.rowptr, hg.col, w, objective=obj)
    wg = pg.weighted_graph(mem, hg.rowptr, hg.col, w, objective=obj)
    return og, wg


def _run_both(mem, hg, obj, method, ex_iters, seed):
    og, wg = _both(mem, hg, obj)
    cd_o = O.ClusterData(og, obj, 1.0)
    cd_g = pg.get_objective(mem, wg, obj, 1.0)
    lo, so = O.run_clustering(og, cd_o, method=method, ex_iters=ex_iters, seed=seed)
    lg, sg = pg.run_clustering(mem, wg, cd_g, method=method, ex_iters=ex_iters, seed=seed)
    q, _ = pg.verify_objective(mem, wg, lg, obj)
    cd_g.close()
    wg.close()
    return lo, so, lg, sg, q


@pytest.mark.parametrize("ex_iters", [0, -1])
def test_planted_sbm_65k_plouvain(mem, ex_iters):
    hg = graph("sbm65k")
    assert hg.n == 65536
    lo, so, lg, sg, q = _run_both(mem, hg, pg.OBJ_MOD, pg.METHOD_LOUVAIN, ex_iters, 1)
    assert np.array_equal(lo, lg)
    assert so.objective == sg["objective"]
    assert so.label_count == sg["label_count"]
    assert so.levels == sg["levels"]
    # the planted 64 blocks are found: 64 clusters, each block's majority
    # label distinct and covering at least 99 % of the block
    assert sg["label_count"] == 64
    maj = []
    for b in range(64):
        cnt = np.bincount(lg[b * 1024:(b + 1) * 1024])
        maj.append(int(cnt.argmax()))
        assert cnt.max() >= 0.99 * 1024
    assert len(set(maj)) == 64
    assert abs(q - sg["objective"]) < 1e-9


def test_dcsbm_4m_pleidenplus_first_pass(mem):
    hg = graph("dcsbm4m")
    assert hg.n == 4194304
    lo, so, lg, sg, q = _run_both(mem, hg, pg.OBJ_WMOD, pg.METHOD_LEIDEN_PLUS, 0, 1)
    assert np.array_equal(lo, lg)
    assert so.objective == sg["objective"]
    assert so.label_count == sg["label_count"]
    assert so.levels == sg["levels"]
    assert abs(q - sg["objective"]) < 1e-9


def test_rmat22_plouvain(mem):
    hg = graph("rmat22")
    assert np.diff(hg.rowptr).max() >= 15000  # massive-bucket rows present
    lo, so, lg, sg, q = _run_both(mem, hg, pg.OBJ_MOD, pg.METHOD_LOUVAIN, 0, 1)
    assert np.array_equal(lo, lg)
    assert so.objective == sg["objective"]
    assert so.label_count == sg["label_count"]
    assert so.levels == sg["levels"]
    assert abs(q - sg["objective"]) < 1e-9


def test_rmat22_level0_contraction(mem):
    """The first level of pLouvain on R-MAT 22: the initial local move, then
    build_coarse_graph of its labels (sorted coarse rows, summed weights)."""
    hg = graph("rmat22")
    og, wg = _both(mem, hg, pg.OBJ_MOD)
    cd_o = O.ClusterData(og, pg.OBJ_MOD, 1.0)
    cd_g = pg.get_objective(mem, wg, pg.OBJ_MOD, 1.0)
    part = np.arange(hg.n, dtype=np.int32)
    po, _, _ = O.local_move(og, cd_o, part, True)
    pgp = part.copy()
    pg.local_move(mem, wg, pgp, cd_g, True)
    assert np.array_equal(po, pgp)
    nc = int(cd_g.label_count)
    assert nc == cd_o.info()["label_count"]
    assert nc > 262144  # above the shared-bitmap placement limit
    co = O.build_coarse_graph(og, po, nc)
    cg = pg.build_coarse_graph(mem, wg, pgp, nc)
    ro, col_o, w_o, vw_o = co.arrays()
    rg, col_g, w_g, vw_g = cg.to_host()
    assert np.array_equal(ro, rg)
    assert np.array_equal(col_o, col_g)
    assert np.array_equal(w_o, w_g)
    assert np.array_equal(vw_o, vw_g)
    # summed weights: the coarse graph keeps the weight of every edge between
    # clusters (unit weights: nnz minus the directed intra-cluster edges)
    assert int(w_g.astype(np.int64).sum()) == hg.nnz - int(cd_g.uncut)
    cd_g.close()
    cg.close()
    wg.close()
