"""GPU graph input against the oracle (oracle/graph_io.py): Matrix Market files
of every banner kind built on the GPU (app/io/io_mtx.cpp:95-345), METIS files
(app/io/io_metis.cpp:64-181), raw edge lists, malformed files, and a clustering
of a loaded graph equal to one of the oracle-built CSR.  Integer work:
bit-exact."""
import numpy as np
import pytest

import pennsylvaniagpugraphclustering_b200 as pg
from oracle import graph_io as GIO

pytestmark = pytest.mark.gpu


def _mtx_text(rng, n, m, field, sym, self_loops=0.05, zero_w=0.05, dup=0.1, comments=True):
    src = rng.integers(0, n, m)
    dst = rng.integers(0, n, m)
    sl = rng.random(m) < self_loops
    dst[sl] = src[sl]
    dp = rng.random(m) < dup
    if m > 1:  # duplicates of earlier entries, some reversed
        j = rng.integers(0, m, m)
        rev = rng.random(m) < 0.5
        src[dp] = np.where(rev[dp], dst[j[dp]], src[j[dp]])
        dst[dp] = np.where(rev[dp], src[j[dp]], dst[j[dp]])
    lines = [f"%%MatrixMarket matrix coordinate {field} {'symmetric' if sym else 'general'}"]
    if comments:
        lines.append("% generated")
    lines.append(f"{n} {n} {m}")
    for k in range(m):
        if field == "pattern":
            lines.append(f"{src[k] + 1} {dst[k] + 1}")
        elif field == "integer":
            w = 0 if rng.random() < zero_w else int(rng.integers(1, 9))
            lines.append(f"{src[k] + 1} {dst[k] + 1} {w}")
        else:
            lines.append(f"{src[k] + 1} {dst[k] + 1} {rng.random():.4f}")
        if comments and k % 97 == 5:
            lines.append("% interleaved comment")
    return ("\n".join(lines) + "\n").encode()


def _metis_text(rng, n, p, weighted):
    a = np.triu(rng.random((n, n)) < p, 1)
    wt = np.triu(rng.integers(1, 20, (n, n)), 1)
    a = a | a.T
    wt = wt + wt.T
    m = int(a.sum()) // 2
    lines = ["% metis", f"{n} {m}" + (" 1" if weighted else "")]
    for i in range(n):
        nb = np.flatnonzero(a[i])
        if weighted:
            lines.append(" ".join(f"{j + 1} {wt[i, j]}" for j in nb))
        else:
            lines.append(" ".join(str(j + 1) for j in nb))
    return ("\n".join(lines) + "\n").encode()


def _check(mem, path, objective):
    wg = pg.load_graph(mem, str(path), objective)
    rp, c, w, _ = wg.to_host()
    erp, ec, ew, euni = GIO.load_graph(str(path), objective)
    assert wg.edge_uniform == euni
    assert np.array_equal(rp, erp)
    assert np.array_equal(c, ec)
    if euni:
        assert w is None
    else:
        assert np.array_equal(w, ew)
    return wg


@pytest.mark.parametrize("field", ["pattern", "integer", "real"])
@pytest.mark.parametrize("sym", [True, False])
@pytest.mark.parametrize("objective", [pg.OBJ_MOD, pg.OBJ_WMOD])
def test_mtx_matches_oracle(mem, tmp_path, field, sym, objective):
    rng = np.random.default_rng(["pattern", "integer", "real"].index(field) * 4 + sym * 2 + objective)
    p = tmp_path / "g.mtx"
    p.write_bytes(_mtx_text(rng, 300, 2500, field, sym))
    _check(mem, p, objective)


def test_mtx_larger_than_one_sort_tile(mem, tmp_path):
    rng = np.random.default_rng(5)
    p = tmp_path / "big.mtx"
    p.write_bytes(_mtx_text(rng, 40000, 300000, "integer", True, comments=False))
    _check(mem, p, pg.OBJ_WMOD)
    p2 = tmp_path / "big_general.mtx"
    p2.write_bytes(_mtx_text(rng, 40000, 300000, "pattern", False, comments=False))
    _check(mem, p2, pg.OBJ_MOD)


def test_mtx_edge_shapes(mem, tmp_path):
    cases = {
        "empty.mtx": b"%%MatrixMarket matrix coordinate pattern symmetric\n0 0 0\n",
        "no_edges.mtx": b"%%MatrixMarket matrix coordinate pattern symmetric\n5 5 0\n",
        "only_loops.mtx": b"%%MatrixMarket matrix coordinate pattern general\n3 3 2\n1 1\n2 2\n",
        "no_newline.mtx": b"%%MatrixMarket matrix coordinate integer symmetric\n2 2 1\n2 1 3",
        "one_vertex.mtx": b"%%MatrixMarket matrix coordinate pattern symmetric\n1 1 1\n1 1\n",
    }
    for name, data in cases.items():
        p = tmp_path / name
        p.write_bytes(data)
        _check(mem, p, pg.OBJ_WMOD)


@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("objective", [pg.OBJ_CPM, pg.OBJ_WMOD])
def test_metis_matches_oracle(mem, tmp_path, weighted, objective):
    rng = np.random.default_rng(7 + weighted)
    p = tmp_path / "g.graph"
    p.write_bytes(_metis_text(rng, 200, 0.05, weighted))
    _check(mem, p, objective)


@pytest.mark.parametrize("name,data", [
    ("a.mtx", b"%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n"),
    ("b.mtx", b"%%MatrixMarket matrix coordinate pattern general\n2 3 1\n1 2\n"),
    ("c.mtx", b"%%MatrixMarket matrix coordinate pattern general\n3 3 2\n1 2\n3\n"),
    ("d.mtx", b"%%MatrixMarket matrix coordinate pattern general\n3 3 3\n1 2\n2 3\n"),
    ("e.mtx", b"%%MatrixMarket matrix coordinate pattern general\n3 3 1\n1 2\n2 3\n"),
    ("f.mtx", b"%%MatrixMarket matrix coordinate pattern general\n3 3 1\n1 4\n"),
    ("g.graph", b"2 1 10\n2 1\n1 1\n"),
    ("h.graph", b"2 1 0 1\n2\n1\n"),
    ("i.graph", b"3 2\n2\n1\n"),
    ("j.graph", b"2 1\n3\n1\n"),
    ("k.graph", b"2 1\n1\n2\n"),  # self loops: rejected by the graph checks
])
def test_malformed_files_raise(mem, tmp_path, name, data):
    p = tmp_path / name
    p.write_bytes(data)
    with pytest.raises(pg.InvalidArgument):
        pg.load_graph(mem, str(p), pg.OBJ_MOD)
    # the context stays usable
    q = tmp_path / "ok.mtx"
    q.write_bytes(b"%%MatrixMarket matrix coordinate pattern symmetric\n2 2 1\n2 1\n")
    assert pg.load_graph(mem, str(q), pg.OBJ_MOD).nnz == 2


def test_missing_file_raises(mem, tmp_path):
    with pytest.raises(pg.InvalidArgument):
        pg.load_graph(mem, str(tmp_path / "absent.mtx"), pg.OBJ_MOD)


@pytest.mark.parametrize("sym", [True, False])
def test_edges_from_host_and_device_match_oracle(mem, sym):
    import torch
    rng = np.random.default_rng(3)
    n, m = 100000, 1500000
    src = rng.integers(0, n, m).astype(np.int32)
    dst = rng.integers(0, n, m).astype(np.int32)
    dst[::50] = src[::50]
    w = rng.integers(0, 6, m).astype(np.int32) if sym else None
    erp, ec, ew = GIO.construct_from_edgelist(n, src, dst, w, sym)
    for dev in (False, True):
        args = (src, dst) if not dev else (torch.from_numpy(src).cuda(), torch.from_numpy(dst).cuda())
        ww = w if (w is None or not dev) else torch.from_numpy(w).cuda()
        wg = pg.graph_from_edges(mem, n, *args, weights=ww, symmetric=sym, objective=pg.OBJ_WMOD)
        rp, c, wo, _ = wg.to_host()
        assert np.array_equal(rp, erp) and np.array_equal(c, ec)
        if sym:
            assert np.array_equal(wo, ew)
        else:
            assert wo is None


def test_edges_reject_bad_ids(mem):
    with pytest.raises(pg.InvalidArgument):
        pg.graph_from_edges(mem, 3, np.array([0, 3], np.int32), np.array([1, 1], np.int32))
    with pytest.raises(pg.InvalidArgument):
        pg.graph_from_edges(mem, 3, np.array([0, -1], np.int32), np.array([1, 1], np.int32))


def test_loaded_graph_clusters_like_the_oracle_csr(mem, tmp_path):
    rng = np.random.default_rng(9)
    p = tmp_path / "g.mtx"
    p.write_bytes(_mtx_text(rng, 3000, 30000, "integer", True, comments=False))
    wg = pg.load_graph(mem, str(p), pg.OBJ_WMOD)
    erp, ec, ew, _ = GIO.load_graph(str(p), pg.OBJ_WMOD)
    wg2 = pg.weighted_graph(mem, erp, ec, ew, objective=pg.OBJ_WMOD)
    out = []
    for g in (wg, wg2):
        cd = pg.get_objective(mem, g, pg.OBJ_WMOD, 1.0)
        labels, st = pg.run_clustering(mem, g, cd, method=pg.METHOD_LEIDEN_PLUS, ex_iters=0, seed=4)
        out.append((labels, st["objective"]))
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]


def test_vertex_weight_file_feeds_the_objective(mem, tmp_path):
    """-vw_file: load_view + load_graph(vtx_w=...) equals the oracle given the
    same weights (CPM, where vertex weights are the cluster sizes)."""
    from oracle import oracle as O
    rng = np.random.default_rng(13)
    p = tmp_path / "g.mtx"
    p.write_bytes(_mtx_text(rng, 2000, 12000, "pattern", True, comments=False))
    vwf = tmp_path / "vw.txt"
    vw = rng.integers(1, 5, 2000).astype(np.int64)
    pg.write_part(vw, vwf)
    vw_in = pg.load_view(2000, vwf)
    assert np.array_equal(vw_in, vw)
    wg = pg.load_graph(mem, str(p), pg.OBJ_CPM, vtx_w=vw_in)
    rp, c, _, vg = wg.to_host()
    assert np.array_equal(vg, vw)
    og = O.Graph(rp, c, None, vtx_w=vw, objective=pg.OBJ_CPM)
    cd_o = O.ClusterData(og, pg.OBJ_CPM, 1.0)
    cd_g = pg.get_objective(mem, wg, pg.OBJ_CPM, 1.0)
    lo, so = O.run_clustering(og, cd_o, method=pg.METHOD_LEIDEN_PLUS, ex_iters=0, seed=2)
    lg, sg = pg.run_clustering(mem, wg, cd_g, method=pg.METHOD_LEIDEN_PLUS, ex_iters=0, seed=2)
    assert np.array_equal(lo, lg) and so.objective == sg["objective"]
    with pytest.raises(ValueError):
        wg.set_vertex_weights(vw[:10])
