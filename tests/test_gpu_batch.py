"""GPU tests of batched clustering (pggc_batch_run): concurrent jobs on several
streams give exactly the results of sequential runs, for a population of
seeds on one graph and for a set of uneven-size graphs."""
import numpy as np
import pytest

import pennsylvaniagpugraphclustering_b200 as pg
from pennsylvaniagpugraphclustering_b200 import graphgen as gg

from . import graphs as G

pytestmark = pytest.mark.gpu


def _seq(mem, g, obj, method, ex_iters, seed):
    cd = pg.get_objective(mem, g, obj, 1.0)
    lab, st = pg.run_clustering(mem, g, cd, method=method, ex_iters=ex_iters, seed=seed)
    return lab, st


def test_batch_population_of_seeds_matches_sequential(mem):
    hg = G.small_dcsbm(seed=5)
    g = pg.weighted_graph(mem, hg.rowptr, hg.col, hg.w, objective=pg.OBJ_WMOD)
    jobs = [dict(graph=g, objective=pg.OBJ_WMOD, method=pg.METHOD_LEIDEN_PLUS, ex_iters=1, seed=s)
            for s in range(1, 9)]
    res = pg.batch_run(mem, jobs, streams=4)
    for j, (lab, st) in zip(jobs, res):
        lo, so = _seq(mem, g, pg.OBJ_WMOD, pg.METHOD_LEIDEN_PLUS, 1, j["seed"])
        assert np.array_equal(lab, lo)
        assert st["objective"] == so["objective"]
        assert st["label_count"] == so["label_count"]


def test_batch_uneven_graphs_matches_sequential(mem):
    rng = np.random.default_rng(7)
    graphs = []
    for k in range(12):
        n = int(np.exp(rng.uniform(np.log(1000), np.log(30000))))
        blocks = int(rng.integers(8, 64))
        hg = gg.sbm(n, blocks, 12.0, 3.0, int(rng.integers(1, 1 << 30)))
        graphs.append(pg.weighted_graph(mem, hg.rowptr, hg.col, None, objective=pg.OBJ_MOD))
    methods = [pg.METHOD_LOUVAIN, pg.METHOD_LEIDEN, pg.METHOD_LEIDEN_PLUS]
    jobs = [dict(graph=g, objective=pg.OBJ_MOD, method=methods[k % 3], ex_iters=0, seed=k + 1)
            for k, g in enumerate(graphs)]
    res = pg.batch_run(mem, jobs, streams=6)
    for j, (lab, st) in zip(jobs, res):
        lo, so = _seq(mem, j["graph"], pg.OBJ_MOD, j["method"], 0, j["seed"])
        assert np.array_equal(lab, lo)
        assert st["objective"] == so["objective"]


def test_batch_reports_the_failing_job(mem):
    hg = G.small_sbm()
    g = pg.weighted_graph(mem, hg.rowptr, hg.col, None, objective=pg.OBJ_MOD)
    jobs = [dict(graph=g, method=pg.METHOD_LEIDEN, seed=1), dict(graph=g, method=7, seed=2)]
    with pytest.raises(Exception) as ei:
        pg.batch_run(mem, jobs, streams=2)
    assert "method" in str(ei.value)
