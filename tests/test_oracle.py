"""CPU tests of the oracle (no GPU).

The reference ships no tests, golden vectors or fixtures and cannot be built
here (Kokkos is absent), so the oracle is pinned against independent
restatements instead: pure-Python transliterations of the reference's per-vertex
rules on small graphs, numpy/scipy computations of the same quantities, the
published MurmurHash3 test vector, and hand-computed known answers.
"""
import numpy as np
import pytest

from oracle import oracle as O

from . import graphs as G

# ---------------------------------------------------------------------------
# hashes and fixed-association arithmetic
# ---------------------------------------------------------------------------


def murmur3_py(key: int) -> int:
    """MurmurHash3_x86_32 (Appleby) of one 4-byte little-endian key, seed 0."""
    M = 0xFFFFFFFF
    rotl = lambda x, r: ((x << r) | (x >> (32 - r))) & M  # noqa: E731
    k = (key * 0xCC9E2D51) & M
    k = rotl(k, 15)
    k = (k * 0x1B873593) & M
    h = k
    h = rotl(h, 13)
    h = (h * 5 + 0xE6546B64) & M
    h ^= 4
    h ^= h >> 16
    h = (h * 0x85EBCA6B) & M
    h ^= h >> 13
    h = (h * 0xC2B2AE35) & M
    h ^= h >> 16
    return h


def test_murmur3_published_vector():
    # MurmurHash3_x86_32 of four zero bytes with seed 0
    assert O.murmur3(0) == 0x2362F9DE


def test_murmur3_matches_python_restatement():
    rng = np.random.default_rng(0)
    for k in rng.integers(0, 2**32, 500):
        assert O.murmur3(int(k)) == murmur3_py(int(k))


def butterfly(v):
    v = list(v)
    d = 16
    while d >= 1:
        v = [v[l] + v[l ^ d] for l in range(32)]
        d >>= 1
    return v[0]


def det_reduce_py(a):
    cur = list(a)
    if not cur:
        return 0.0
    while True:
        nxt = []
        for g in range(0, len(cur), 32):
            grp = cur[g:g + 32] + [0.0] * (32 - len(cur[g:g + 32]))
            nxt.append(butterfly(grp))
        cur = nxt
        if len(cur) == 1:
            return cur[0]


def det_scan_py(a):
    k = len(a)
    out = [0.0] * k
    groups = (k + 31) // 32
    tot = []
    for g in range(groups):
        v = [a[g * 32 + l] if g * 32 + l < k else 0.0 for l in range(32)]
        d = 1
        while d < 32:
            v = [v[l] + v[l - d] if l >= d else v[l] for l in range(32)]
            d <<= 1
        for l in range(32):
            if g * 32 + l < k:
                out[g * 32 + l] = v[l]
        tot.append(v[31])
    if groups > 1:
        S = det_scan_py(tot)
        for g in range(1, groups):
            for l in range(32):
                i = g * 32 + l
                if i < k:
                    out[i] = S[g - 1] + out[i]
    return out


@pytest.mark.parametrize("k", [1, 5, 32, 33, 1000, 1025, 40000])
def test_det_reduce_and_scan_association(k):
    rng = np.random.default_rng(k)
    a = rng.standard_normal(k) * 10.0 ** rng.integers(-8, 8, k)
    assert O.det_reduce(a) == det_reduce_py(a.tolist())
    if k <= 1025:
        assert np.array_equal(O.det_scan(a), np.array(det_scan_py(a.tolist())))


def test_det_scan_exact_on_integers():
    a = np.arange(100000, dtype=np.float64) % 97
    assert np.array_equal(O.det_scan(a), np.cumsum(a))


# ---------------------------------------------------------------------------
# ordering, contraction, objective
# ---------------------------------------------------------------------------


@pytest.mark.parametrize("mk", [G.small_rmat, G.hub_graph, G.two_cliques])
def test_orderings_against_numpy(mk):
    g = mk()
    deg = np.diff(g.rowptr)
    b1 = np.where(deg < 128, 0, np.where(deg < 15000, 1, 2))
    b2 = np.where(deg < 64, 0, np.where(deg < 15000, 1, 2))
    o1, o2, off = O.generate_orderings(g.rowptr)
    assert np.array_equal(o1, np.argsort(b1, kind="stable"))
    assert np.array_equal(o2, np.argsort(b2, kind="stable"))
    assert off[0] == (b1 == 0).sum() and off[1] == (b1 < 2).sum()
    assert off[2] == (b2 == 0).sum() and off[3] == off[1]


def _coarse_numpy(g, vcmap, nc, weighted):
    import scipy.sparse as sp
    src = np.repeat(np.arange(g.n), np.diff(g.rowptr))
    w = g.w.astype(np.float64) if weighted else np.ones(g.nnz)
    cu, cv = vcmap[src], vcmap[g.col]
    keep = cu != cv
    M = sp.coo_matrix((w[keep], (cu[keep], cv[keep])), shape=(nc, nc)).tocsr()
    M.sum_duplicates()
    M.sort_indices()
    return M


@pytest.mark.parametrize("weighted", [False, True])
def test_contraction_against_scipy(weighted):
    g = G.small_dcsbm(n=5000)
    og = O.Graph(g.rowptr, g.col, g.w if weighted else None, objective=O.OBJ_WMOD if weighted else O.OBJ_MOD)
    rng = np.random.default_rng(1)
    nc = 700
    vcmap = rng.integers(0, nc, g.n).astype(np.int32)
    vcmap[:nc] = np.arange(nc)
    cg = O.build_coarse_graph(og, vcmap, nc)
    rowptr, col, w, vw = cg.arrays()
    M = _coarse_numpy(g, vcmap, nc, weighted)
    assert np.array_equal(rowptr, M.indptr)
    assert np.array_equal(col, M.indices)
    if weighted:
        assert np.array_equal(w, M.data.astype(np.float32))
    else:
        assert np.array_equal(w, M.data.astype(np.int32))
    _, _, _, fvw = og.arrays()
    expect = np.zeros(nc, fvw.dtype)
    np.add.at(expect, vcmap, fvw)
    assert np.array_equal(vw, expect)


def modularity_numpy(g, labels, weighted):
    src = np.repeat(np.arange(g.n), np.diff(g.rowptr))
    w = g.w.astype(np.float64) if weighted else np.ones(g.nnz)
    deg = np.zeros(g.n)
    np.add.at(deg, src, w)
    two_m = w.sum()
    uncut = w[labels[src] == labels[g.col]].sum()
    D = np.zeros(g.n)
    np.add.at(D, labels, deg)
    return (uncut - (D * D).sum() / two_m) / two_m


@pytest.mark.parametrize("weighted", [False, True])
def test_verify_objective_against_numpy(weighted):
    g = G.small_dcsbm(n=3000)
    og = O.Graph(g.rowptr, g.col, g.w if weighted else None, objective=O.OBJ_WMOD if weighted else O.OBJ_MOD)
    labels = np.random.default_rng(2).integers(0, 40, g.n).astype(np.int32)
    q, _ = O.verify_objective(og, labels, O.OBJ_WMOD if weighted else O.OBJ_MOD)
    assert abs(q - modularity_numpy(g, labels, weighted)) < 1e-9


# ---------------------------------------------------------------------------
# the local-move rules against a pure-Python transliteration
# ---------------------------------------------------------------------------


def f32(x):
    return np.float32(x)


def select_py(g, vw, part, pvals, D, lam, fr, initial, dest_in):
    """src/local_mover.cpp:474-515 (thread path) with ties -> smallest cluster id."""
    n = g.n
    pm = f32(lam)
    dest = dest_in.copy()
    gain = np.zeros(n, np.float32)
    for i in range(n):
        if dest[i] == O.NO_MOVE:
            continue
        w = int(vw[i])
        multi = f32(f32(w) * pm)
        p = int(part[i])
        p_conn = f32(f32(pvals[i]) - f32(f32(int(D[p]) - w) * multi))
        thr = f32(0.0) if p_conn < 0 else f32(float(p_conn) * (1.0 - float(f32(fr))))
        conn = {}
        for j in range(g.rowptr[i], g.rowptr[i + 1]):
            v = int(g.col[j])
            c = v if initial else int(part[v])
            if not initial and c == p:
                continue
            conn[c] = conn.get(c, 0) + 1
        best, bc = None, None
        for c, jv in conn.items():
            if not (jv > 0 and f32(jv) >= thr):
                continue
            jc = f32(f32(jv) - f32(f32(int(D[c])) * multi))
            if jc >= thr and (best is None or jc > bc or (jc == bc and c < best)):
                best, bc = c, jc
        if best is not None:
            dest[i], gain[i] = best, f32(bc - p_conn)
        elif p_conn < 0:
            dest[i], gain[i] = O.NEW_PART, f32(-p_conn)
        else:
            dest[i], gain[i] = O.NO_MOVE, np.finfo(np.float32).min
    return dest, gain


@pytest.mark.parametrize("initial", [True, False])
@pytest.mark.parametrize("fr", [0.0, 0.25, 0.75])
def test_select_against_python(initial, fr):
    g = G.ring_of_cliques(12, 6)
    og = O.Graph(g.rowptr, g.col, objective=O.OBJ_MOD)
    cd = O.ClusterData(og, O.OBJ_MOD, 1.0)
    _, _, _, vw = og.arrays()
    n = g.n
    if initial:
        part = np.arange(n, dtype=np.int32)
        pv = np.zeros(n, np.int64)
        D = vw.copy()
    else:
        rng = np.random.default_rng(3)
        L = 15
        part = rng.integers(0, L, n).astype(np.int32)
        part[:L] = np.arange(L)
        D = np.zeros(L, np.int64)
        np.add.at(D, part, vw)
        src = np.repeat(np.arange(n), np.diff(g.rowptr))
        pv = np.zeros(n, np.int64)
        np.add.at(pv, src[part[src] == part[g.col]], 1)
        cd.set_state(D, pv.sum())
    dest0 = np.full(n, O.NULL_PART, np.int32)
    lam = cd.info()["lambda"]
    do, go, _ = O.select(og, cd, part, pv, dest0, fr, initial)
    dp, gp = select_py(g, vw, part, pv, D, lam, fr, initial, dest0)
    assert np.array_equal(do, dp)
    assert np.array_equal(go, gp)


# ---------------------------------------------------------------------------
# known answers and invariants of the full methods
# ---------------------------------------------------------------------------


@pytest.mark.parametrize("method", [O.METHOD_LOUVAIN, O.METHOD_LEIDEN, O.METHOD_LEIDEN_PLUS])
def test_two_cliques_known_answer(method):
    g = G.two_cliques(6)
    og = O.Graph(g.rowptr, g.col, objective=O.OBJ_MOD)
    cd = O.ClusterData(og, O.OBJ_MOD, 1.0)
    labels, st = O.run_clustering(og, cd, method=method)
    assert len(np.unique(labels)) == 2
    assert len(np.unique(labels[:6])) == 1 and len(np.unique(labels[6:])) == 1
    # uncut 60 of 62 directed edges, both clusters have volume 31: Q = 29/62
    assert abs(st.objective - 29.0 / 62.0) < 1e-12


def test_planted_partition_recovered():
    from pennsylvaniagpugraphclustering_b200 import graphgen as gg
    g = gg.planted_sbm_65k(1)
    og = O.Graph(g.rowptr, g.col, objective=O.OBJ_MOD)
    cd = O.ClusterData(og, O.OBJ_MOD, 1.0)
    labels, st = O.run_clustering(og, cd, method=O.METHOD_LOUVAIN)
    blocks = np.arange(g.n) // 1024
    majority = []
    for b in range(64):
        vals, cnt = np.unique(labels[blocks == b], return_counts=True)
        assert cnt.max() >= 0.99 * 1024
        majority.append(vals[cnt.argmax()])
    assert len(set(majority)) == 64
    q, _ = O.verify_objective(og, labels, O.OBJ_MOD)
    assert abs(q - st.objective) < 1e-12


@pytest.mark.parametrize("seed", [1, 2])
def test_leiden_clusters_connected(seed):
    g = G.small_rmat(seed=seed, scale=11)
    og = O.Graph(g.rowptr, g.col, objective=O.OBJ_MOD)
    cd = O.ClusterData(og, O.OBJ_MOD, 1.0)
    labels, _ = O.run_clustering(og, cd, method=O.METHOD_LEIDEN, seed=seed)
    assert O.connected_components(g.rowptr, g.col, labels) == len(np.unique(labels))


def test_local_move_monotone():
    g = G.small_dcsbm(n=4000)
    og = O.Graph(g.rowptr, g.col, g.w, objective=O.OBJ_WMOD)
    cd = O.ClusterData(og, O.OBJ_WMOD, 1.0)
    part = np.arange(g.n, dtype=np.int32)
    last = cd.info()["obj"]
    for limit in (1, 2, 3):
        cd2 = O.ClusterData(og, O.OBJ_WMOD, 1.0)
        _, st, _ = O.local_move(og, cd2, part, True, sweep_limit=limit)
        assert st.raw_obj >= last
        last = st.raw_obj


def objective_numpy(g, w, vw, labels, objective, mult):
    """The objectives of interface/cluster_data.hpp:38-181 in closed form:
    obj = uncut - lambda * sum_c vol(c)^2 with the subclass's lambda and
    normalisation (Mod/WMod: lambda = mult / g_deg, objective = obj / g_deg;
    CPM: lambda = mult / 2, objective = obj + lambda * n; NLCC: lambda =
    mult * g_deg / vol^2, objective = obj / g_deg; LCC: lambda = mult)."""
    src = np.repeat(np.arange(g.n), np.diff(g.rowptr))
    ww = np.ones(g.nnz) if w is None else w.astype(np.float64)
    uncut = ww[labels[src] == labels[g.col]].sum()
    vol = np.zeros(g.n)
    np.add.at(vol, labels, vw.astype(np.float64))
    sq = (vol * vol).sum()
    g_deg = float(g.nnz) if w is None else ww.sum()
    if objective in (O.OBJ_MOD, O.OBJ_WMOD):
        gd = float(g.nnz) if objective == O.OBJ_MOD else vw.astype(np.float64).sum()
        lam = mult / gd
        return (uncut - lam * sq) / gd
    if objective == O.OBJ_CPM:
        lam = mult * 0.5
        return uncut - lam * sq + lam * g.n
    if objective == O.OBJ_NLCC:
        vt = vw.astype(np.float64).sum()
        lam = mult * g_deg / (vt * vt)
        return (uncut - lam * sq) / g_deg
    return uncut - mult * sq


@pytest.mark.parametrize("objective", [O.OBJ_CPM, O.OBJ_NLCC, O.OBJ_LCC])
@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("mult", [1.0, 0.3])
def test_other_objectives_against_closed_form(objective, weighted, mult):
    """CPM, NLCC and LCC values of the oracle (int32 weights) against the
    closed forms of the reference's cluster_data subclasses, with the default
    unit vertex weights and with custom ones."""
    g = G.small_dcsbm(n=3000)
    w = np.maximum(np.rint(g.w.astype(np.float64) * 4), 1).astype(np.int32) if weighted else None
    labels = np.random.default_rng(7).integers(0, 60, g.n).astype(np.int32)
    uses_w = weighted and objective not in (O.OBJ_CPM,)
    for vw in (None, np.random.default_rng(3).integers(1, 9, g.n).astype(np.int64)):
        og = O.Graph(g.rowptr, g.col, w if uses_w else None, vtx_w=vw, objective=objective)
        q, _ = O.verify_objective(og, labels, objective, mult)
        vw_eff = np.ones(g.n, np.int64) if vw is None else vw
        ref = objective_numpy(g, w if uses_w else None, vw_eff, labels, objective, mult)
        assert abs(q - ref) <= 1e-9 * max(1.0, abs(ref))


# ---------------------------------------------------------------------------
# one whole sweep (select, afterburner, moves, best-state relabel) against a
# pure-Python transliteration of src/local_mover.cpp:280-433 and :1361-1417
# ---------------------------------------------------------------------------


def xorshift32(x):
    x &= 0xFFFFFFFF
    x ^= (x << 13) & 0xFFFFFFFF
    x ^= x >> 17
    x ^= (x << 5) & 0xFFFFFFFF
    return x


def as_i32(x):
    return x - (1 << 32) if x >= (1 << 31) else x


def canon_sum_py(terms):
    """32-lane strided accumulation from 0.0, then the xor butterfly."""
    v = [0.0] * 32
    for k, t in enumerate(terms):
        v[k & 31] = v[k & 31] + t
    for d in (16, 8, 4, 2, 1):
        v = [v[l] + v[l ^ d] for l in range(32)]
    return v[0]


def afterburner_py(g, vw, part, dest, gain, lam):
    eps = f32(0.1)
    pm = f32(lam)
    keep = {}
    for i in range(g.n):
        best = int(dest[i])
        if best == O.NO_MOVE:
            continue
        p = int(part[i])
        multi = f32(f32(int(vw[i])) * pm)
        igain = f32(gain[i])
        hi = as_i32(xorshift32(i))
        terms = []
        for j in range(g.rowptr[i], g.rowptr[i + 1]):
            v = int(g.col[j])
            d = f32(f32(gain[v]) - igain)
            if d >= eps or (abs(d) < eps and as_i32(xorshift32(v)) < hi):
                q = f32(f32(1.0) - f32(multi * f32(int(vw[v]))))
                coef = 0
                if int(dest[v]) == p:
                    coef -= 1
                if int(dest[v]) == best and best != O.NEW_PART:
                    coef += 1
                if int(part[v]) == p:
                    coef += 1
                if int(part[v]) == best:
                    coef -= 1
                terms.append(float(coef) * float(q))
            else:
                terms.append(0.0)
        keep[i] = f32(igain + f32(canon_sum_py(terms))) >= 0
    return keep


@pytest.mark.parametrize("graph", ["ring", "sbm"])
def test_first_sweep_against_python(graph):
    """Singletons, one annealed sweep (filter ratio 0.75): the oracle's best
    partition equals the transliteration's moved partition, relabelled in
    label order, when the sweep raises modularity."""
    g = G.ring_of_cliques(12, 6) if graph == "ring" else G.from_edges(
        200, [tuple(e) for e in np.random.default_rng(5).integers(0, 200, (700, 2)) if e[0] != e[1]])
    if graph == "sbm":  # the edge list may hold duplicates: keep the first of each pair
        src = np.repeat(np.arange(g.n), np.diff(g.rowptr))
        keep = np.ones(g.nnz, bool)
        keep[1:] = (src[1:] != src[:-1]) | (g.col[1:] != g.col[:-1])
        src, col = src[keep], g.col[keep]
        rowptr = np.zeros(g.n + 1, np.int64)
        np.add.at(rowptr, src + 1, 1)
        g = G.HostGraph(np.cumsum(rowptr), col.astype(np.int32), None, name="random")
    og = O.Graph(g.rowptr, g.col, objective=O.OBJ_MOD)
    cd = O.ClusterData(og, O.OBJ_MOD, 1.0)
    _, _, _, vw = og.arrays()
    n = g.n
    lam = cd.info()["lambda"]
    part = np.arange(n, dtype=np.int32)
    dest, gain = select_py(g, vw, part, np.zeros(n, np.int64), vw.copy(), lam, 0.75, True,
                           np.full(n, O.NULL_PART, np.int32))
    keep = afterburner_py(g, vw, part, dest, gain, lam)
    moved = part.copy()
    for i, k in keep.items():
        if k:
            moved[i] = dest[i]
    q_before, _ = O.verify_objective(og, part, O.OBJ_MOD)
    q_after, _ = O.verify_objective(og, moved, O.OBJ_MOD)
    out, _, _ = O.local_move(og, cd, part, True, enable_sa=True, sweep_limit=1)
    if q_after > q_before:
        _, expect = np.unique(moved, return_inverse=True)
        assert np.array_equal(out, expect.astype(np.int32))
    else:
        assert np.array_equal(out, part)


# ---------------------------------------------------------------------------
# coarsen_leidenR (src/leidenR.cpp:41-500, unit weights) against a pure-Python
# transliteration
# ---------------------------------------------------------------------------


def c_mod(a, b):
    """C's % on signed operands (the remainder takes the dividend's sign)."""
    r = abs(a) % abs(b)
    return -r if a < 0 else r


def leidenR_py(g, vw, constraint, td, lam, seed_pick, seed_order):
    n = g.n
    SPLIT = 1000000000
    ORD_MAX = 2147483647
    gamma = f32(lam)
    src = np.repeat(np.arange(n), np.diff(g.rowptr))
    pv = np.zeros(n, np.int64)
    np.add.at(pv, src[constraint[src] == constraint[g.col]], 1)
    well = [f32(int(pv[i])) >= f32(f32(gamma * f32(int(vw[i]))) * f32(int(td[constraint[i]]) - int(vw[i])))
            for i in range(n)]
    hn = list(range(n))
    for i in range(n):
        b, e = int(g.rowptr[i]), int(g.rowptr[i + 1])
        width = e - b
        multi = f32(gamma * f32(int(vw[i])))
        jxs = as_i32(murmur3_py((seed_pick + i) & 0xFFFFFFFF))
        if c_mod(jxs, 1000) == 0 or not well[i] or width == 0:
            continue
        jx = b + (jxs & 0xFFFFFFFF) % width
        for s in range(width):
            j = jx + s
            if j >= e:
                j -= width
            v = int(g.col[j])
            if constraint[i] != constraint[v] or not well[v]:
                continue
            if f32(1.0) >= f32(multi * f32(int(vw[v]))):
                hn[i] = v
                break
    order = [abs(c_mod(as_i32(murmur3_py((i + seed_order) & 0xFFFFFFFF)), SPLIT)) for i in range(n)]
    for i in range(n):
        if order[i] == order[hn[i]]:
            hn[i] = i
    vcmap = [ORD_MAX] * n
    for i in range(n):  # find_trees, src/leidenR.cpp:213-260
        now, then = i, hn[i]
        if now == then:
            vcmap[i] = i
            continue
        while order[now] > order[then]:
            now, then = then, hn[then]
        if now != i:
            vcmap[i] = now
            vcmap[now] = now
    for i in range(n):
        if vcmap[i] == ORD_MAX:
            order[i] = 2 * SPLIT - order[i]
    unassigned = [vcmap[i] == ORD_MAX for i in range(n)]
    for i in range(n):
        if not unassigned[i]:
            continue
        now, then = i, hn[i]
        while vcmap[now] == ORD_MAX and order[now] > order[then]:
            now, then = then, hn[then]
        vcmap[i] = vcmap[now]
    # ensure_gamma_connectivity, src/leidenR.cpp:41-187
    ids = sorted(range(n), key=lambda a: (vcmap[a], order[a], a))
    start = {}
    for x, i in enumerate(ids):
        start.setdefault(vcmap[i], x)
    ts, s = [0] * n, 0
    for x, i in enumerate(ids):
        ts[x] = s
        s += int(vw[i])
    inner = [0] * n
    for i in range(n):
        for j in range(g.rowptr[i], g.rowptr[i + 1]):
            v = int(g.col[j])
            if vcmap[i] == vcmap[v] and order[v] < order[i]:
                inner[i] += 1
    breakers = {}
    for x, i in enumerate(ids):
        c = vcmap[i]
        prev = ts[x] - ts[start[c]]
        if f32(inner[i]) < f32(f32(gamma * f32(int(vw[i]))) * f32(prev)):
            breakers[c] = min(breakers.get(c, n), x)
    oc, s = [0] * n, 0
    for x, i in enumerate(ids):
        s += int(pv[i]) - 2 * inner[i]
        oc[i] = s
    for x, i in enumerate(ids):
        c = vcmap[i]
        cb = start[c]
        curr = ts[x] + int(vw[i]) - ts[cb]
        other = int(td[constraint[i]]) - curr
        outer = oc[i] - (oc[ids[cb - 1]] if cb > 0 else 0)
        if f32(outer) < f32(f32(gamma * f32(curr)) * f32(other)):
            breakers[c] = min(breakers.get(c, n), x + 1)
    for x, i in enumerate(ids):
        if x >= breakers.get(vcmap[i], n):
            vcmap[i] = i
    nc = 0  # contigitize, src/leidenR.cpp:190-210
    for u in range(n):
        if vcmap[u] == u:
            vcmap[u] = nc
            nc += 1
        else:
            vcmap[u] += n
    for u in range(n):
        if vcmap[u] >= n:
            vcmap[u] = vcmap[vcmap[u] - n]
    return np.array(vcmap, np.int32), nc


@pytest.mark.parametrize("seeds", [(1, 2), (12345, 678), (0xDEADBEEF, 0x12345678)])
def test_leidenR_against_python(seeds):
    g = G.small_sbm()
    og = O.Graph(g.rowptr, g.col, objective=O.OBJ_MOD)
    cd = O.ClusterData(og, O.OBJ_MOD, 1.0)
    _, _, _, vw = og.arrays()
    louv, _, _ = O.local_move(og, cd, np.arange(g.n, dtype=np.int32), True)
    td = cd.total_deg()
    vo, nco = O.coarsen_leidenR(og, cd, louv, *seeds)
    vp, ncp = leidenR_py(g, vw, louv, td, cd.info()["lambda"], *seeds)
    assert nco == ncp
    assert np.array_equal(vo, vp)
    assert 0 < nco < g.n
