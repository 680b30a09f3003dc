"""Error paths of the C ABI on the GPU: invalid inputs are rejected before any
kernel indexes with them, and a device-side bounded loop that gives up returns
PGGC_ERR_DEVICE while the context stays usable.  Nothing here faults, traps or
hangs the GPU: failures are injected from the host."""
import numpy as np
import pytest

import pennsylvaniagpugraphclustering_b200 as pg
from pennsylvaniagpugraphclustering_b200 import _lib

from . import graphs as G

pytestmark = pytest.mark.gpu


def test_self_loop_rejected(mem):
    g = G.from_edges(3, [(0, 1), (1, 2)])
    col = g.col.copy()
    col[0] = 0  # row 0 now points to itself
    with pytest.raises(pg.InvalidArgument):
        pg.weighted_graph(mem, g.rowptr, col)


def test_column_out_of_range_rejected(mem):
    g = G.from_edges(3, [(0, 1), (1, 2)])
    col = g.col.copy()
    col[-1] = 7
    with pytest.raises(pg.InvalidArgument):
        pg.weighted_graph(mem, g.rowptr, col)


def test_bad_rowptr_rejected(mem):
    g = G.from_edges(3, [(0, 1), (1, 2)])
    rp = g.rowptr.copy()
    rp[1], rp[2] = rp[2], rp[1]
    with pytest.raises(pg.InvalidArgument):
        pg.weighted_graph(mem, rp, g.col)


def test_labels_out_of_range_rejected(mem):
    g = G.two_cliques()
    wg = pg.weighted_graph(mem, g.rowptr, g.col)
    bad = np.zeros(g.n, np.int32)
    bad[3] = g.n + 5
    with pytest.raises(pg.InvalidArgument):
        pg.build_coarse_graph(mem, wg, bad, 2)
    cd = pg.get_objective(mem, wg, pg.OBJ_MOD)
    with pytest.raises(pg.InvalidArgument):
        pg.clustering_methods.leiden_part(mem, wg, cd, input=bad, improve=True)


def test_probe_limit_gives_device_error_and_context_recovers(mem):
    g = G.small_sbm()
    wg = pg.weighted_graph(mem, g.rowptr, g.col)
    # 512 coarse vertices of ~8 scattered members: each hashes ~100 distinct
    # neighbour ids from [0, 512) into 256 slots, so single-probe inserts collide
    nc = 512
    part = ((np.arange(g.n, dtype=np.int64) * 7919) % nc).astype(np.int32)
    cd = pg.get_objective(mem, wg, pg.OBJ_MOD)
    _lib.check(_lib.lib().pggc_debug_set_probe_limit(mem.handle, 1))
    try:
        with pytest.raises(pg.DeviceError):
            pg.build_coarse_graph(mem, wg, part, nc)
    finally:
        _lib.check(_lib.lib().pggc_debug_set_probe_limit(mem.handle, 0))
    cg = pg.build_coarse_graph(mem, wg, part, nc)
    assert cg.n == nc and cg.nnz > 0
    labels, st = pg.run_clustering(mem, wg, cd, method=pg.METHOD_LOUVAIN)
    assert st["label_count"] >= 1


def test_destruction_order_is_free(mem):
    """Graphs and cluster data may outlive the Python context object."""
    m2 = pg.memory_store(0)
    g = G.two_cliques()
    wg = pg.weighted_graph(m2, g.rowptr, g.col)
    cd = pg.get_objective(m2, wg, pg.OBJ_MOD)
    m2.close()  # the C context stays alive while wg and cd reference it
    cd.close()
    wg.close()
