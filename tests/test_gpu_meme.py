"""GPU parity of the memetic driver (app/memetic_clustering.cpp:27-219) with the
oracle: intersection ids, cut-edge signatures, and whole runs with a fixed
offspring count (same random stream on both sides)."""
import numpy as np
import pytest

import pennsylvaniagpugraphclustering_b200 as pg
from oracle import oracle as O

from . import graphs as G

pytestmark = pytest.mark.gpu


def test_intersection_matches_oracle(mem):
    rng = np.random.default_rng(11)
    for n, k1, k2 in [(1, 1, 1), (1000, 7, 300), (50000, 900, 1200)]:
        c1 = rng.integers(0, k1, n).astype(np.int32)
        c2 = rng.integers(0, k2, n).astype(np.int32)
        go, gk = pg.intersect_clusters(mem, c1, c2)
        oo, ok = O.intersect(c1, c2)
        assert gk == ok
        assert np.array_equal(go, oo)


@pytest.mark.parametrize("name", ["sbm", "hub", "dcsbm"])
def test_signature_matches_oracle(mem, name):
    hg = {"sbm": G.small_sbm, "hub": G.hub_graph, "dcsbm": G.small_dcsbm}[name]()
    wg = pg.weighted_graph(mem, hg.rowptr, hg.col, None, objective=pg.OBJ_MOD)
    og = O.Graph(hg.rowptr, hg.col)
    lab = np.random.default_rng(2).integers(0, max(hg.n // 10, 1), hg.n).astype(np.int32)
    assert np.array_equal(pg.cut_signature(mem, wg, lab), O.signature(og, lab))


@pytest.mark.parametrize("name,obj", [("sbm", pg.OBJ_MOD), ("dcsbm", pg.OBJ_WMOD)])
def test_meme_cluster_matches_oracle(mem, name, obj):
    hg = {"sbm": G.small_sbm, "dcsbm": G.small_dcsbm}[name]()
    w = None if obj == pg.OBJ_MOD else hg.w
    wg = pg.weighted_graph(mem, hg.rowptr, hg.col, w, objective=obj)
    og = O.Graph(hg.rowptr, hg.col, w, objective=obj)
    lg, sg = pg.meme_cluster(mem, wg, obj, pop_size=4, offspring=5, seed=21)
    lo, so = O.meme_cluster(og, obj, pop_size=4, offspring=5, seed=21)
    assert np.array_equal(lg, lo)
    assert sg["objective"] == so.objective
    assert sg["replaced"] == so.replaced
    assert sg["best_initial"] == so.best_initial
    assert sg["objective"] >= sg["best_initial"]


def test_meme_rejects_bad_arguments(mem):
    hg = G.small_sbm()
    wg = pg.weighted_graph(mem, hg.rowptr, hg.col, None, objective=pg.OBJ_MOD)
    with pytest.raises(Exception):
        pg.meme_cluster(mem, wg, pg.OBJ_MOD, pop_size=1, offspring=1)
    with pytest.raises(Exception):
        pg.meme_cluster(mem, wg, pg.OBJ_MOD, pop_size=4, offspring=-1, time_limit_s=0.0)
