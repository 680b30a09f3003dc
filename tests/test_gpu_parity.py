"""GPU parity: every hot-path function through the C ABI against the CPU oracle.

Integer and FP32-weighted graphs are compared bit-exactly: both sides use the
same canonical arithmetic (FP32 gain expressions operation by operation, int64
or FP64 sums in a fixed association, smallest-id tie breaks, sorted coarse rows,
MurmurHash3 random picks), so any difference is a bug.
"""
import numpy as np
import pytest

import pennsylvaniagpugraphclustering_b200 as pg
from oracle import oracle as O

from . import graphs as G

pytestmark = pytest.mark.gpu


def _pair(mem, hg, objective):
    uniform = objective in (pg.OBJ_MOD, pg.OBJ_CPM) or hg.w is None
    w = None if uniform else hg.w
    vw = getattr(hg, "vw", None)
    if vw is not None and (w is None or w.dtype != np.float32):
        vw = vw.astype(np.int64) if vw.dtype != np.int64 else vw
    og = O.Graph(hg.rowptr, hg.col, w, vtx_w=vw, objective=objective)
    wg = pg.weighted_graph(mem, hg.rowptr, hg.col, w, objective=objective, vtx_w=vw)
    return og, wg


CASES = [
    ("two_cliques", G.two_cliques, pg.OBJ_MOD),
    ("ring_of_cliques", G.ring_of_cliques, pg.OBJ_MOD),
    ("star", G.star, pg.OBJ_MOD),
    ("path", G.path, pg.OBJ_MOD),
    ("isolated", G.with_isolated, pg.OBJ_MOD),
    ("sbm", G.small_sbm, pg.OBJ_MOD),
    ("rmat12", G.small_rmat, pg.OBJ_MOD),
    ("dcsbm_wmod", G.small_dcsbm, pg.OBJ_WMOD),
    ("dcsbm_mod", G.small_dcsbm, pg.OBJ_MOD),
    ("hub_wmod", G.hub_graph, pg.OBJ_WMOD),
    ("hub_mod", G.hub_graph, pg.OBJ_MOD),
    # the other objectives (interface/cluster_data.hpp:109-181)
    ("sbm_cpm", G.small_sbm, pg.OBJ_CPM),
    ("hub_cpm", G.hub_graph, pg.OBJ_CPM),
    ("dcsbm_nlcc", G.small_dcsbm, pg.OBJ_NLCC),
    ("dcsbm_lcc", G.small_dcsbm, pg.OBJ_LCC),
    ("hub_lcc", G.hub_graph, pg.OBJ_LCC),
    # int32 edge weights, the reference's weight type
    ("dcsbm_int_wmod", lambda: G.int_weighted(G.small_dcsbm()), pg.OBJ_WMOD),
    ("dcsbm_int_nlcc", lambda: G.int_weighted(G.small_dcsbm()), pg.OBJ_NLCC),
    ("hub_int_nlcc", lambda: G.int_weighted(G.hub_graph()), pg.OBJ_NLCC),
    # custom vertex weights (app/io/vertex_weighting.cpp:27-42 replaced by the caller's)
    ("sbm_mod_vw", lambda: G.with_vertex_weights(G.small_sbm(), 1), pg.OBJ_MOD),
    ("dcsbm_wmod_vw", lambda: G.with_vertex_weights(G.small_dcsbm(), 2), pg.OBJ_WMOD),
    ("rmat_cpm_vw", lambda: G.with_vertex_weights(G.small_rmat(), 3), pg.OBJ_CPM),
]
IDS = [c[0] for c in CASES]

_CACHE = {}


def case_graph(name):
    if name not in _CACHE:
        for nm, fn, obj in CASES:
            if nm == name:
                _CACHE[name] = (fn(), obj)
    return _CACHE[name]


@pytest.mark.parametrize("name", IDS)
def test_vertex_weights_and_objective(mem, name):
    hg, obj = case_graph(name)
    og, wg = _pair(mem, hg, obj)
    _, _, _, vw_o = og.arrays()
    _, _, _, vw_g = wg.to_host()
    assert np.array_equal(vw_o, vw_g)
    cd_o = O.ClusterData(og, obj, 1.0)
    cd_g = pg.get_objective(mem, wg, obj, 1.0)
    io = cd_o.info()
    assert io["lambda"] == cd_g.lambda_
    assert io["obj"] == cd_g.obj
    assert io["label_count"] == cd_g.label_count


@pytest.mark.parametrize("name", IDS)
def test_generate_orderings(mem, name):
    hg, obj = case_graph(name)
    og, wg = _pair(mem, hg, obj)
    o1, o2, off = O.generate_orderings(hg.rowptr)
    g1, g2, goff = pg.generate_orderings(mem, wg)
    assert np.array_equal(o1, g1)
    assert np.array_equal(o2, g2)
    assert np.array_equal(off, goff)


def _random_map(n, nc, seed):
    rng = np.random.default_rng(seed)
    m = rng.integers(0, nc, n).astype(np.int32)
    m[:nc] = np.arange(nc, dtype=np.int32)  # every coarse id used
    return m


@pytest.mark.parametrize("name", IDS)
@pytest.mark.parametrize("ratio", [2, 7])
def test_build_coarse_graph(mem, name, ratio):
    hg, obj = case_graph(name)
    og, wg = _pair(mem, hg, obj)
    nc = max(1, hg.n // ratio)
    vcmap = _random_map(hg.n, nc, ratio)
    co = O.build_coarse_graph(og, vcmap, nc)
    cg = pg.build_coarse_graph(mem, wg, vcmap, nc)
    ro, col_o, w_o, vw_o = co.arrays()
    rg, col_g, w_g, vw_g = cg.to_host()
    assert np.array_equal(ro, rg)
    assert np.array_equal(col_o, col_g)
    assert np.array_equal(w_o, w_g)
    assert np.array_equal(vw_o, vw_g)
    # rows sorted, no self loops
    for c in range(min(nc, 200)):
        row = col_g[rg[c]:rg[c + 1]]
        assert np.all(np.diff(row) > 0)
        assert not np.any(row == c)


@pytest.mark.parametrize("name", IDS)
@pytest.mark.parametrize("fr", [0.0, 0.25, 0.75])
@pytest.mark.parametrize("initial", [True, False])
def test_select_pass(mem, name, fr, initial):
    hg, obj = case_graph(name)
    og, wg = _pair(mem, hg, obj)
    n = hg.n
    cd_o = O.ClusterData(og, obj, 1.0)
    cd_g = pg.get_objective(mem, wg, obj, 1.0)
    if initial:
        part = np.arange(n, dtype=np.int32)
        pv = np.zeros(n, wg.vdtype)
    else:
        # a coarse random partition with its exact state
        L = max(1, n // 5)
        part = _random_map(n, L, 11)
        _, _, w, vw = og.arrays()
        td = np.zeros(L, wg.vdtype)
        np.add.at(td, part, vw)
        src = np.repeat(np.arange(n), np.diff(hg.rowptr))
        same = part[src] == part[hg.col]
        ww = np.ones(hg.nnz) if w is None else w.astype(np.float64)
        pv = np.zeros(n, np.float64)
        np.add.at(pv, src[same], ww[same])
        pv = pv.astype(wg.vdtype)
        uncut = pv.sum()
        cd_o.set_state(td, uncut)
        cd_g.set_state(L, td, uncut)
    dest0 = np.full(n, pg.NULL_PART, np.int32)
    dest0[::7] = pg.NO_MOVE
    gain0 = np.linspace(-1, 1, n).astype(np.float32)
    do, go, ko = O.select(og, cd_o, part, pv, dest0, fr, initial, gain=gain0)
    dg, gg_, kg = pg.select_pass(mem, wg, cd_g, part, pv, dest0, fr, initial, gain=gain0)
    assert np.array_equal(go[::7], gain0[::7])
    assert ko == kg
    assert np.array_equal(do, dg)
    assert np.array_equal(go.view(np.int32), gg_.view(np.int32))


@pytest.mark.parametrize("name", IDS)
@pytest.mark.parametrize("limit", [1, 2, -1])
def test_local_move_initial(mem, name, limit):
    hg, obj = case_graph(name)
    og, wg = _pair(mem, hg, obj)
    n = hg.n
    cd_o = O.ClusterData(og, obj, 1.0)
    cd_g = pg.get_objective(mem, wg, obj, 1.0)
    part = np.arange(n, dtype=np.int32)
    po, st, _ = O.local_move(og, cd_o, part, True, enable_sa=True, sweep_limit=limit)
    pgp = part.copy()
    pg.local_move(mem, wg, pgp, cd_g, True, sweep_limit=limit)
    assert np.array_equal(po, pgp)
    io = cd_o.info()
    assert io["label_count"] == cd_g.label_count
    assert io["obj"] == cd_g.obj
    assert np.array_equal(cd_o.total_deg(), cd_g.total_deg())


@pytest.mark.parametrize("name", IDS)
@pytest.mark.parametrize("strict", [False, True])
def test_local_move_from_partition(mem, name, strict):
    """Non-initial call (conn tables built from an existing partition), SA off / strict."""
    hg, obj = case_graph(name)
    og, wg = _pair(mem, hg, obj)
    n = hg.n
    cd_o = O.ClusterData(og, obj, 1.0)
    cd_g = pg.get_objective(mem, wg, obj, 1.0)
    part = np.arange(n, dtype=np.int32)
    po, _, _ = O.local_move(og, cd_o, part, True, sweep_limit=2)
    pgp = part.copy()
    pg.local_move(mem, wg, pgp, cd_g, True, sweep_limit=2)
    assert np.array_equal(po, pgp)
    po2, _, _ = O.local_move(og, cd_o, po, False, enable_sa=False, strict=strict)
    pg2 = pgp.copy()
    if strict:
        pg.local_move_strict(mem, wg, pg2, cd_g, False)
    else:
        pg.local_move(mem, wg, pg2, cd_g, False, enable_simulated_annealing=False)
    assert np.array_equal(po2, pg2)
    assert cd_o.info()["obj"] == cd_g.obj
    assert cd_o.info()["label_count"] == cd_g.label_count


@pytest.mark.parametrize("name", IDS)
def test_coarsen_leidenR(mem, name):
    hg, obj = case_graph(name)
    og, wg = _pair(mem, hg, obj)
    n = hg.n
    cd_o = O.ClusterData(og, obj, 1.0)
    cd_g = pg.get_objective(mem, wg, obj, 1.0)
    part = np.arange(n, dtype=np.int32)
    po, _, _ = O.local_move(og, cd_o, part, True)
    pgp = part.copy()
    pg.local_move(mem, wg, pgp, cd_g, True)
    assert np.array_equal(po, pgp)
    for seeds in [(1, 2), (12345, 678), (0xDEADBEEF, 0x12345678)]:
        vo, nco = O.coarsen_leidenR(og, cd_o, po, *seeds)
        vg, ncg = pg.coarsen_leidenR(mem, wg, pgp, cd_g, *seeds)
        assert nco == ncg
        assert np.array_equal(vo, vg)


@pytest.mark.parametrize("name", IDS)
@pytest.mark.parametrize("method", [pg.METHOD_LOUVAIN, pg.METHOD_LEIDEN, pg.METHOD_LEIDEN_PLUS])
def test_run_clustering(mem, name, method):
    hg, obj = case_graph(name)
    og, wg = _pair(mem, hg, obj)
    cd_o = O.ClusterData(og, obj, 1.0)
    cd_g = pg.get_objective(mem, wg, obj, 1.0)
    lo, so = O.run_clustering(og, cd_o, method=method, ex_iters=0, seed=7)
    lg, sg = pg.run_clustering(mem, wg, cd_g, method=method, ex_iters=0, seed=7)
    assert np.array_equal(lo, lg)
    assert so.objective == sg["objective"]
    assert so.label_count == sg["label_count"]
    assert so.levels == sg["levels"]
    if method == pg.METHOD_LEIDEN:
        # every pLeiden cluster is connected
        assert O.connected_components(hg.rowptr, hg.col, lg) == len(np.unique(lg))


@pytest.mark.parametrize("name", ["sbm", "dcsbm_wmod", "rmat12"])
def test_run_clustering_ex_iters(mem, name):
    hg, obj = case_graph(name)
    og, wg = _pair(mem, hg, obj)
    cd_o = O.ClusterData(og, obj, 1.0)
    cd_g = pg.get_objective(mem, wg, obj, 1.0)
    lo, so = O.run_clustering(og, cd_o, method=pg.METHOD_LEIDEN_PLUS, ex_iters=-1, seed=3)
    lg, sg = pg.run_clustering(mem, wg, cd_g, method=pg.METHOD_LEIDEN_PLUS, ex_iters=-1, seed=3)
    assert np.array_equal(lo, lg)
    assert so.objective == sg["objective"]


@pytest.mark.parametrize("name", IDS)
def test_verify_objective(mem, name):
    hg, obj = case_graph(name)
    og, wg = _pair(mem, hg, obj)
    labels = _random_map(hg.n, max(1, hg.n // 9), 5)
    vo, ro = O.verify_objective(og, labels, obj)
    vg, rg = pg.verify_objective(mem, wg, labels, obj)
    assert vo == vg and ro == rg


@pytest.mark.parametrize("weighted", [False, True])
def test_build_coarse_graph_row_wider_than_shared_table(mem, weighted):
    """A coarse row with ~40,000 distinct neighbours: more than a 16,384-slot
    shared table holds, so the row takes the global-table fallback."""
    leaves = 40000
    rng = np.random.default_rng(4)
    w = rng.uniform(0.5, 1.5, leaves).astype(np.float32) if weighted else None
    hg = G.from_edges(leaves + 1, [(0, i) for i in range(1, leaves + 1)], w)
    obj = pg.OBJ_WMOD if weighted else pg.OBJ_MOD
    og, wg = _pair(mem, hg, obj)
    vcmap = np.concatenate([[0, 0], np.arange(1, leaves, dtype=np.int32)]).astype(np.int32)
    nc = leaves
    co = O.build_coarse_graph(og, vcmap, nc)
    cg = pg.build_coarse_graph(mem, wg, vcmap, nc)
    for a, b in zip(co.arrays(), cg.to_host()):
        assert np.array_equal(a, b)
    rg = cg.to_host()[0]
    assert rg[1] - rg[0] == leaves - 1


@pytest.mark.parametrize("weighted", [False, True])
def test_select_pass_vertex_wider_than_shared_table(mem, weighted):
    """A 40,000-degree hub whose neighbours are all in distinct clusters: more
    candidate clusters than a 16,384-slot shared table holds, so the hub takes
    the global-table pass."""
    leaves = 40000
    rng = np.random.default_rng(9)
    w = rng.uniform(0.5, 1.5, leaves).astype(np.float32) if weighted else None
    hg = G.from_edges(leaves + 1, [(0, i) for i in range(1, leaves + 1)], w)
    obj = pg.OBJ_WMOD if weighted else pg.OBJ_MOD
    og, wg = _pair(mem, hg, obj)
    n = hg.n
    cd_o = O.ClusterData(og, obj, 1.0)
    cd_g = pg.get_objective(mem, wg, obj, 1.0)
    part = np.arange(n, dtype=np.int32)
    _, _, _, vw = og.arrays()
    td = vw.astype(wg.vdtype)
    pv = np.zeros(n, wg.vdtype)
    cd_o.set_state(td, 0)
    cd_g.set_state(n, td, 0)
    dest0 = np.full(n, pg.NULL_PART, np.int32)
    gain0 = np.zeros(n, np.float32)
    for fr in (0.0, 0.75):
        do, go, ko = O.select(og, cd_o, part, pv, dest0, fr, False, gain=gain0)
        dg, gg_, kg = pg.select_pass(mem, wg, cd_g, part, pv, dest0, fr, False, gain=gain0)
        assert ko == kg
        assert np.array_equal(do, dg)
        assert np.array_equal(go.view(np.int32), gg_.view(np.int32))


def test_int_weighted_lcc_louvain(mem):
    """LCC on int32 weights 2..6 at lambda 1: pLouvain parity.  (pLeiden on this
    graph reaches a level where the refinement contracts nothing while the
    local move still merges; the reference's level loop has no bound there, and
    both sides stop with an error after 4096 levels.)"""
    hg = G.int_weighted(G.small_dcsbm(n=5000))
    og, wg = _pair(mem, hg, pg.OBJ_LCC)
    cd_o = O.ClusterData(og, pg.OBJ_LCC, 1.0)
    cd_g = pg.get_objective(mem, wg, pg.OBJ_LCC, 1.0)
    lo, so = O.run_clustering(og, cd_o, method=pg.METHOD_LOUVAIN, ex_iters=0, seed=7)
    lg, sg = pg.run_clustering(mem, wg, cd_g, method=pg.METHOD_LOUVAIN, ex_iters=0, seed=7)
    assert np.array_equal(lo, lg)
    assert so.objective == sg["objective"] and so.label_count == sg["label_count"]


@pytest.mark.parametrize("weighted", [False, True])
def test_build_coarse_graph_above_bitmap_limit(mem, weighted):
    """More coarse vertices than the shared-bitmap placement covers (262,144):
    the comparison-sort placement kernels (register, warp rank, block bitonic,
    radix for long rows) against the oracle."""
    hg = G.small_rmat(seed=4, scale=19)
    if weighted:
        hg = G.HostGraph(hg.rowptr, hg.col, G.symmetric_weights(hg), name="rmat19w")
    obj = pg.OBJ_WMOD if weighted else pg.OBJ_MOD
    og, wg = _pair(mem, hg, obj)
    for nc, seed in ((300000, 1), (270000, 2)):
        vcmap = _random_map(hg.n, nc, seed)
        # a few heavy coarse vertices: rows long enough for the block and radix paths
        vcmap[: hg.n // 64] = np.arange(hg.n // 64, dtype=np.int32) % 8
        co = O.build_coarse_graph(og, vcmap, nc)
        cg = pg.build_coarse_graph(mem, wg, vcmap, nc)
        ro, col_o, w_o, vw_o = co.arrays()
        rg, col_g, w_g, vw_g = cg.to_host()
        assert np.array_equal(ro, rg)
        assert np.array_equal(col_o, col_g)
        assert np.array_equal(w_o, w_g)
        assert np.array_equal(vw_o, vw_g)


@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("fr", [0.0, 0.75])
def test_select_pass_hub_row_at_unaligned_offset(mem, weighted, fr):
    """A 40,000-leaf hub whose row starts 6 edges into the column array (not on
    a 16-byte boundary) and ends on a ragged tail: the split select stages
    each 8192-edge chunk with a bulk copy of its aligned middle and plain loads
    of the rest; the result must equal the oracle's."""
    leaves = 40000
    edges = [(0, 1), (1, 2), (0, 2)] + [(3, 4 + k) for k in range(leaves)]
    rng = np.random.default_rng(21)
    w = rng.uniform(0.5, 1.5, len(edges)).astype(np.float32) if weighted else None
    hg = G.from_edges(4 + leaves, edges, w)
    assert hg.rowptr[3] % 4 != 0 and hg.rowptr[4] % 4 != 0
    obj = pg.OBJ_WMOD if weighted else pg.OBJ_MOD
    og, wg = _pair(mem, hg, obj)
    n = hg.n
    cd_o = O.ClusterData(og, obj, 1.0)
    cd_g = pg.get_objective(mem, wg, obj, 1.0)
    part = np.arange(n, dtype=np.int32)
    _, _, _, vw = og.arrays()
    td = vw.astype(wg.vdtype)
    pv = np.zeros(n, wg.vdtype)
    cd_o.set_state(td, 0)
    cd_g.set_state(n, td, 0)
    dest0 = np.full(n, pg.NULL_PART, np.int32)
    gain0 = np.zeros(n, np.float32)
    do, go, ko = O.select(og, cd_o, part, pv, dest0, fr, False, gain=gain0)
    dg, gg_, kg = pg.select_pass(mem, wg, cd_g, part, pv, dest0, fr, False, gain=gain0)
    assert ko == kg
    assert np.array_equal(do, dg)
    assert np.array_equal(go.view(np.int32), gg_.view(np.int32))


@pytest.mark.parametrize("weighted", [False, True])
def test_build_coarse_graph_wide_row_at_unaligned_offset(mem, weighted):
    """The 40,000-neighbour coarse row is the fourth coarse vertex, so its flat
    member-edge list starts 3 entries in (not on a 16-byte boundary): the split
    contraction stages its chunks by bulk copies of the aligned middle and
    plain loads of the rest."""
    leaves = 40000
    rng = np.random.default_rng(5)
    w = rng.uniform(0.5, 1.5, leaves).astype(np.float32) if weighted else None
    hg = G.from_edges(leaves + 1, [(0, i) for i in range(1, leaves + 1)], w)
    obj = pg.OBJ_WMOD if weighted else pg.OBJ_MOD
    og, wg = _pair(mem, hg, obj)
    vcmap = np.empty(leaves + 1, np.int32)
    vcmap[0] = 3
    vcmap[1:4] = [0, 1, 2]
    vcmap[4] = 3
    vcmap[5:] = np.arange(4, leaves, dtype=np.int32)
    nc = leaves
    co = O.build_coarse_graph(og, vcmap, nc)
    cg = pg.build_coarse_graph(mem, wg, vcmap, nc)
    for x, y in zip(co.arrays(), cg.to_host()):
        assert np.array_equal(x, y)
    rg = cg.to_host()[0]
    assert rg[4] - rg[3] == leaves - 1


@pytest.mark.parametrize("extra", [1000, 270000])
def test_build_coarse_graph_row_sizes_at_sort_boundaries(mem, extra):
    """Stars whose centres become coarse rows of exactly u distinct columns,
    for u around every boundary of the placement sorts (32-key chunks, the
    warp's 256, the block's 1024), leaves mapped to shuffled coarse ids; with
    1,000 or 270,000 further isolated vertices, so the coarse graph is below
    or above the bitmap placement's 262,144 vertices."""
    sizes = [31, 32, 33, 63, 64, 65, 100, 255, 256, 257, 511, 512, 513, 1000, 1023, 1024, 1025]
    edges, v = [], 0
    for u in sizes:
        c = v
        edges += [(c, c + 1 + k) for k in range(u)]
        v += u + 1
    n = v + extra
    rng = np.random.default_rng(17)
    w = rng.uniform(0.5, 1.5, len(edges)).astype(np.float32)
    hg = G.from_edges(n, edges, w)
    og, wg = _pair(mem, hg, pg.OBJ_WMOD)
    vcmap = rng.permutation(n).astype(np.int32)  # every vertex its own coarse vertex, shuffled ids
    co = O.build_coarse_graph(og, vcmap, n)
    cg = pg.build_coarse_graph(mem, wg, vcmap, n)
    for x, y in zip(co.arrays(), cg.to_host()):
        assert np.array_equal(x, y)
    rg = cg.to_host()[0]
    deg = np.diff(rg)
    for u in sizes:
        assert (deg == u).any()


@pytest.mark.parametrize("weighted", [False, True])
def test_build_coarse_graph_member_layouts(mem, weighted):
    """Coarse rows assembled from awkward member lists: members without edges
    (isolated vertices) between real ones, a coarse vertex with no members,
    rows of many members, and an overflowing row made of ~20,000 members."""
    base = G.small_rmat(seed=5, scale=17)
    iso = 3000
    rowptr = np.concatenate([base.rowptr, np.full(iso, base.rowptr[-1], np.int64)])
    w = G.symmetric_weights(base) if weighted else None
    hg = G.HostGraph(rowptr, base.col, w, name="rmat17+isolated")
    n0, n = base.n, hg.n
    obj = pg.OBJ_WMOD if weighted else pg.OBJ_MOD
    og, wg = _pair(mem, hg, obj)
    rng = np.random.default_rng(13)
    for nc in (300, 3000, 40000):
        vcmap = rng.integers(1, nc, n).astype(np.int32)  # coarse vertex 0 has no members
        vcmap[n0:n0 + 2000] = 2                          # 2000 isolated members ...
        vcmap[40000:40100] = 2                           # ... around 100 real ones
        vcmap[50000:53000] = 5                           # 3000 members
        if nc == 40000:
            vcmap[:20000] = 1                            # the R-MAT hubs: an overflowing row
        co = O.build_coarse_graph(og, vcmap, nc)
        cg = pg.build_coarse_graph(mem, wg, vcmap, nc)
        for x, y in zip(co.arrays(), cg.to_host()):
            assert np.array_equal(x, y)
        rg = cg.to_host()[0]
        assert rg[1] == rg[0] == 0
        if nc == 40000:
            assert rg[2] - rg[1] > 16384


@pytest.mark.parametrize("sizes", [[5000, 500, 30, 10, 3], [20000, 700, 12]])
def test_coarsen_leidenR_tree_sizes(mem, sizes):
    """Disjoint stars: the refinement's trees have ~every star's size, so the
    per-tree sorts run in registers (<= 16 members), per block (<= 1024 and
    <= 16384) and, with a 20,000-leaf star, fall back to the radix sort of all
    vertices."""
    edges, v = [], 0
    for sz in sizes:
        c = v
        edges += [(c, c + 1 + k) for k in range(sz)]
        v += sz + 1
    hg = G.from_edges(v, edges)
    og, wg = _pair(mem, hg, pg.OBJ_MOD)
    cd_o = O.ClusterData(og, pg.OBJ_MOD, 1.0)
    cd_g = pg.get_objective(mem, wg, pg.OBJ_MOD, 1.0)
    part = np.arange(v, dtype=np.int32)
    po, _, _ = O.local_move(og, cd_o, part, True)
    pgp = part.copy()
    pg.local_move(mem, wg, pgp, cd_g, True)
    assert np.array_equal(po, pgp)
    for seeds in [(1, 2), (12345, 678)]:
        vo, nco = O.coarsen_leidenR(og, cd_o, po, *seeds)
        vg, ncg = pg.coarsen_leidenR(mem, wg, pgp, cd_g, *seeds)
        assert nco == ncg
        assert np.array_equal(vo, vg)
    assert np.bincount(vo).max() >= sizes[0] - 30


@pytest.mark.parametrize("weighted", [False, True])
def test_build_coarse_graph_dense_rows(mem, weighted):
    """A graph with long rows (9,000 vertices, mean degree ~145, the shape of
    the coarse levels): the warp-per-vertex flattening, with 300 coarse
    vertices the dense-table hashing and with 9,000 the hash tables."""
    rng = np.random.default_rng(23)
    n, m = 9000, 1300000
    src = rng.integers(0, n, m)
    dst = rng.integers(0, n, m)
    keep = src < dst
    pairs = np.unique(np.stack([src[keep], dst[keep]], axis=1), axis=0)
    edges = list(map(tuple, pairs.tolist()))
    w = rng.uniform(0.5, 1.5, len(edges)).astype(np.float32) if weighted else None
    hg = G.from_edges(n, edges, w)
    assert hg.nnz >= 128 * n
    obj = pg.OBJ_WMOD if weighted else pg.OBJ_MOD
    og, wg = _pair(mem, hg, obj)
    for nc in (300, 9000):
        vcmap = rng.integers(0, nc, n).astype(np.int32)
        vcmap[:nc] = np.arange(nc, dtype=np.int32)
        co = O.build_coarse_graph(og, vcmap, nc)
        cg = pg.build_coarse_graph(mem, wg, vcmap, nc)
        for x, y in zip(co.arrays(), cg.to_host()):
            assert np.array_equal(x, y)
