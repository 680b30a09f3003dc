"""Seeded generators: canonical symmetric CSR, deterministic, workload shapes."""
import numpy as np
import pytest

from pennsylvaniagpugraphclustering_b200 import graphgen as gg


def check_csr(g):
    n = g.n
    assert g.rowptr[0] == 0 and g.rowptr[-1] == g.nnz
    assert np.all(np.diff(g.rowptr) >= 0)
    src = np.repeat(np.arange(n), np.diff(g.rowptr))
    assert np.all((g.col >= 0) & (g.col < n))
    assert not np.any(src == g.col), "self-loop"
    # sorted, no duplicates within rows
    same_row = src[1:] == src[:-1]
    assert np.all(g.col[1:][same_row] > g.col[:-1][same_row])
    # symmetric (with symmetric weights)
    key = src * n + g.col
    rkey = g.col.astype(np.int64) * n + src
    order = np.argsort(key)
    rorder = np.argsort(rkey)
    assert np.array_equal(key[order], rkey[rorder])
    if g.w is not None:
        assert np.array_equal(g.w[order], g.w[rorder])


@pytest.mark.parametrize("make", [
    lambda: gg.sbm(5000, 10, 12.0, 3.0, 3),
    lambda: gg.sbm(5000, 10, 12.0, 3.0, 3, weighted=True),
    lambda: gg.dcsbm(30000, 2),
    lambda: gg.rmat(12, 8, seed=5),
])
def test_canonical_csr(make):
    check_csr(make())


def test_deterministic():
    a, b = gg.dcsbm(20000, 9), gg.dcsbm(20000, 9)
    assert np.array_equal(a.rowptr, b.rowptr) and np.array_equal(a.col, b.col) and np.array_equal(a.w, b.w)
    c = gg.dcsbm(20000, 10)
    assert not (c.nnz == a.nnz and np.array_equal(c.col, a.col))


def test_planted_sbm_shape():
    g = gg.planted_sbm_65k(1)
    assert g.n == 65536
    assert 620_000 < g.m < 690_000  # expected 64*8192 + 131k
    assert abs(np.diff(g.rowptr).mean() - 20.0) < 0.5


def test_dcsbm_shape_scaled():
    g = gg.dcsbm(262144, 1)
    deg = np.diff(g.rowptr)
    assert 17.0 < deg.mean() < 21.0
    assert deg.min() >= 1
    assert g.w.min() >= 0.5 and g.w.max() < 1.5


def test_sbm_population_shapes():
    params = gg.sbm_population_params(256, 1)
    assert len(params) == 256
    ns = np.array([p[0] for p in params])
    bs = np.array([p[1] for p in params])
    assert ns.min() >= 1000 and ns.max() <= 200000
    assert np.all(bs >= 1) and np.all(bs <= 512) and np.all(ns // bs >= 16)
    # log-uniform sizes: about half the graphs below the geometric midpoint
    mid = np.sqrt(1000 * 200000)
    assert 0.35 < np.mean(ns < mid) < 0.65
    assert params == gg.sbm_population_params(256, 1)
    pop = gg.sbm_population(3, 2)
    for g, (n, b, s) in zip(pop, gg.sbm_population_params(3, 2)):
        assert g.n == n
        check_csr(g)
