"""The graph-input oracle (oracle/graph_io.py) on hand-computed cases: the
Matrix Market and METIS rules of app/io/io_mtx.cpp and app/io/io_metis.cpp."""
import numpy as np
import pytest

from oracle import graph_io as GIO


def _csr(rowptr, col, w=None):
    return np.asarray(rowptr, np.int64), np.asarray(col, np.int32), None if w is None else np.asarray(w, np.int32)


def test_mtx_symmetric_integer_weights_kept_for_wmod():
    data = b"%%MatrixMarket matrix coordinate integer symmetric\n% comment\n4 4 4\n2 1 5\n3 1 7\n4 3 2\n4 4 9\n"
    n, s, d, w, sym, uni = GIO.parse_mtx(data, uniform=False)
    assert (n, sym, uni) == (4, True, False)
    rp, c, wo = GIO.construct_from_edgelist(n, s, d, w, sym)
    erp, ec, ew = _csr([0, 2, 3, 5, 6], [1, 2, 0, 0, 3, 2], [5, 7, 5, 7, 2, 2])
    assert np.array_equal(rp, erp) and np.array_equal(c, ec) and np.array_equal(wo, ew)


def test_mtx_weights_ignored_for_mod_and_zero_weight_kept_then():
    data = b"%%MatrixMarket matrix coordinate integer symmetric\n3 3 2\n2 1 0\n3 2 4\n"
    n, s, d, w, sym, uni = GIO.parse_mtx(data, uniform=True)
    assert w is None and uni
    rp, c, _ = GIO.construct_from_edgelist(n, s, d, w, sym)
    assert np.array_equal(rp, [0, 1, 3, 4]) and np.array_equal(c, [1, 0, 2, 1])
    # weighted: the zero-weight entry is dropped
    n, s, d, w, sym, uni = GIO.parse_mtx(data, uniform=False)
    rp, c, wo = GIO.construct_from_edgelist(n, s, d, w, sym)
    assert np.array_equal(rp, [0, 0, 1, 2]) and np.array_equal(c, [2, 1]) and np.array_equal(wo, [4, 4])


def test_mtx_general_is_symmetrised_and_deduplicated():
    data = b"%%MatrixMarket matrix coordinate real general\n3 3 5\n1 2 0.5\n2 1 1.5\n2 3 2.0\n3 3 1.0\n1 2 3\n"
    n, s, d, w, sym, uni = GIO.parse_mtx(data, uniform=False)
    assert not sym and uni and w is None
    rp, c, _ = GIO.construct_from_edgelist(n, s, d, w, sym)
    assert np.array_equal(rp, [0, 1, 3, 4]) and np.array_equal(c, [1, 0, 2, 1])


def test_mtx_real_symmetric_weights_ignored_and_pattern_uniform():
    data = b"%%MatrixMarket matrix coordinate real symmetric\n2 2 1\n2 1 0.25"
    n, s, d, w, sym, uni = GIO.parse_mtx(data, uniform=False)  # no trailing newline
    assert uni and w is None and sym
    data = b"%%MatrixMarket matrix coordinate pattern symmetric\n3 3 2\n2 1\n3 1\n"
    n, s, d, w, sym, uni = GIO.parse_mtx(data, uniform=False)
    assert uni and w is None
    rp, c, _ = GIO.construct_from_edgelist(n, s, d, w, sym)
    assert np.array_equal(rp, [0, 2, 3, 4]) and np.array_equal(c, [1, 2, 0, 0])


@pytest.mark.parametrize("data", [
    b"%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n",  # not coordinate
    b"%%MatrixMarket matrix coordinate pattern general\n2 3 1\n1 2\n",  # bipartite
    b"%%MatrixMarket matrix coordinate pattern general\n3 3 2\n1 2\n3\n",  # one value on a line
    b"%%MatrixMarket matrix coordinate pattern general\n3 3 3\n1 2\n2 3\n",  # too few entries
    b"%%MatrixMarket matrix coordinate pattern general\n3 3 1\n1 2\n2 3\n",  # too many entries
    b"%%MatrixMarket matrix coordinate pattern general\n3 3 1\n1 4\n",  # index out of range
])
def test_mtx_malformed(data):
    with pytest.raises(ValueError):
        n, s, d, w, sym, uni = GIO.parse_mtx(data, uniform=True)


def test_metis_unweighted_and_weighted():
    data = b"% c\n4 3\n2 3\n1\n1 4\n3\n"
    rp, c, w, uni = GIO.parse_metis(data, uniform=True)
    assert uni and w is None
    assert np.array_equal(rp, [0, 2, 3, 5, 6]) and np.array_equal(c, [1, 2, 0, 0, 3, 2])
    data = b"3 2 1\n2 5 3 6\n1 5\n1 6\n"
    rp, c, w, uni = GIO.parse_metis(data, uniform=False)
    assert not uni and np.array_equal(w, [5, 6, 5, 6]) and np.array_equal(c, [1, 2, 0, 0])
    rp, c, w, uni = GIO.parse_metis(data, uniform=True)
    assert uni and w is None and np.array_equal(rp, [0, 2, 3, 4])


def test_metis_isolated_vertex_line_and_comment_between_rows():
    data = b"3 1\n2\n1\n% isolated next\n\n"
    rp, c, w, uni = GIO.parse_metis(data, uniform=True)
    assert np.array_equal(rp, [0, 1, 2, 2]) and np.array_equal(c, [1, 0])


@pytest.mark.parametrize("data", [
    b"2 1 10\n2 1\n1 1\n",  # vertex weights
    b"2 1 0 1\n2\n1\n",  # ncon
    b"3 2\n2\n1\n",  # too few lines / entries
    b"2 1\n3\n1\n",  # neighbour out of range
])
def test_metis_malformed(data):
    with pytest.raises(ValueError):
        GIO.parse_metis(data, uniform=True)


def test_load_graph_dispatches_on_suffix(tmp_path):
    p = tmp_path / "g.mtx"
    p.write_bytes(b"%%MatrixMarket matrix coordinate pattern symmetric\n2 2 1\n2 1\n")
    rp, c, w, uni = GIO.load_graph(str(p), GIO.OBJ_MOD)
    assert np.array_equal(rp, [0, 1, 2]) and np.array_equal(c, [1, 0]) and uni
    p = tmp_path / "g.graph"
    p.write_bytes(b"2 1\n2\n1\n")
    rp, c, w, uni = GIO.load_graph(str(p), GIO.OBJ_WMOD)
    assert np.array_equal(rp, [0, 1, 2]) and np.array_equal(c, [1, 0]) and uni
