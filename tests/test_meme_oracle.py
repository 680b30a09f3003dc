"""CPU checks of the oracle's memetic-driver pieces against independent numpy
restatements (app/memetic_clustering.cpp:27-116)."""
import numpy as np

from oracle import oracle as O

from . import graphs as G


def test_intersection_ranks_distinct_pairs():
    rng = np.random.default_rng(3)
    n = 5000
    c1 = rng.integers(0, 40, n).astype(np.int32)
    c2 = rng.integers(0, 25, n).astype(np.int32)
    out, k = O.intersect(c1, c2)
    pairs = sorted(set(zip(c1.tolist(), c2.tolist())))
    rank = {p: r for r, p in enumerate(pairs)}
    assert k == len(pairs)
    assert np.array_equal(out, np.array([rank[(a, b)] for a, b in zip(c1, c2)], np.int32))
    # vertices share an intersection id exactly when both parents agree
    i, j = rng.integers(0, n, 2000), rng.integers(0, n, 2000)
    assert np.array_equal(out[i] == out[j], (c1[i] == c1[j]) & (c2[i] == c2[j]))


def test_signature_marks_cut_edges():
    hg = G.small_sbm()
    og = O.Graph(hg.rowptr, hg.col)
    rng = np.random.default_rng(5)
    lab = rng.integers(0, 30, hg.n).astype(np.int32)
    sig = O.signature(og, lab)
    src = np.repeat(np.arange(hg.n), np.diff(hg.rowptr))
    cut = lab[src] != lab[hg.col]
    bits = np.zeros(len(sig) * 32, bool)
    bits[:hg.nnz] = cut
    expect = np.packbits(bits.reshape(-1, 32)[:, ::-1], axis=1).view(">u4").ravel().astype(np.uint32)
    assert np.array_equal(sig, expect)


def test_meme_cluster_improves_or_keeps_the_best_initial():
    hg = G.small_sbm()
    og = O.Graph(hg.rowptr, hg.col, objective=O.OBJ_MOD)
    lab, st = O.meme_cluster(og, O.OBJ_MOD, pop_size=4, offspring=4, seed=9)
    assert st.offspring == 4
    assert st.objective >= st.best_initial
    q, _ = O.verify_objective(og, lab, O.OBJ_MOD)
    assert abs(q - st.objective) < 1e-9
