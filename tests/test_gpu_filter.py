"""GPU tests of the learned move filter: the network's kernels against the CPU
oracle (oracle/mlp_oracle.py), sample logging, and the filter inside
clustering runs.

Tolerances: the GPU computes in FP32 (tensor-core products of BF16 operands
for inference, CUDA-core FP32 for training) while the oracle computes the
same rounded network in FP64, so values agree to FP32 accumulation error;
a BF16 rounding of a layer-1 activation that lands on the other side of a
rounding boundary moves a logit by one BF16 step of that activation, which
the inference test allows for a small fraction of rows.
"""
import time

import numpy as np
import pytest

import pennsylvaniagpugraphclustering_b200 as pg
from pennsylvaniagpugraphclustering_b200 import move_filter as MF
from oracle import mlp_oracle as M
from oracle import oracle as O

from . import graphs as G

pytestmark = pytest.mark.gpu


def _features(n, seed):
    rng = np.random.default_rng(seed)
    x = np.stack([rng.uniform(0, 0.7, n), rng.uniform(0, 1, n), rng.uniform(-4, 4, n),
                  (rng.random(n) < 0.3).astype(np.float64), rng.uniform(0, 1, n), rng.uniform(0, 0.2, n),
                  rng.integers(0, 6, n) / 16.0, rng.integers(0, 6, n) / 8.0], axis=1).astype(np.float32)
    return x


def _teacher_labels(x, seed):
    rng = np.random.default_rng(seed)
    score = 1.5 * x[:, 3] - 1.2 * x[:, 1] + 0.4 * x[:, 2] + 0.3 * rng.standard_normal(len(x))
    return (score > 0.2).astype(np.float32)


def test_mlp_infer_matches_oracle(mem):
    p = M.init_params(11)
    p[M.O_B1:M.O_W2] = 0.1
    x = _features(5000, 1)
    lg = MF.infer(mem, p, x)
    ref, _ = M.forward(p, x)
    err = np.abs(lg - ref) / (1.0 + np.abs(ref))
    assert np.quantile(err, 0.99) < 1e-5
    assert err.max() < 2e-2


def test_mlp_infer_edge_counts(mem):
    p = M.init_params(2)
    for n in (1, 31, 32, 33, 1000):
        x = _features(n, n)
        lg = MF.infer(mem, p, x)
        ref, _ = M.forward(p, x)
        assert lg.shape == (n,)
        assert np.all(np.abs(lg - ref) <= 2e-2 * (1.0 + np.abs(ref)))


@pytest.mark.parametrize("n,pos_w", [(1, 1.0), (777, 1.0), (4096, 5.0)])
def test_mlp_loss_grad_matches_oracle(mem, n, pos_w):
    p = M.init_params(5)
    p[M.O_B1:M.O_W2] = 0.05
    x = _features(n, 2)
    y = _teacher_labels(x, 3)
    loss, g = MF.loss_grad(mem, p, x, y, pos_w)
    loss_o, g_o = M.loss_and_grad(p, x, y, pos_w)
    assert abs(loss - loss_o) <= 1e-5 * (1.0 + abs(loss_o))
    scale = np.abs(g_o).max()
    assert np.abs(g - g_o).max() <= 1e-3 * scale + 1e-7


def test_mlp_loss_grad_deterministic(mem):
    p = M.init_params(6)
    x = _features(3000, 4)
    y = _teacher_labels(x, 5)
    l1, g1 = MF.loss_grad(mem, p, x, y, 2.0)
    l2, g2 = MF.loss_grad(mem, p, x, y, 2.0)
    assert l1 == l2 and np.array_equal(g1, g2)


def test_mlp_train_learns_and_is_deterministic(mem):
    x = _features(20000, 7)
    y = _teacher_labels(x, 8)
    p0 = M.init_params(9)
    p1, losses = MF.train(mem, p0, x, y, epochs=6, batch=1024, lr=3e-3, pos_weight=1.0, seed=3)
    p2, _ = MF.train(mem, p0, x, y, epochs=6, batch=1024, lr=3e-3, pos_weight=1.0, seed=3)
    assert np.array_equal(p1, p2)
    assert losses[-1] < losses[0]
    xt = _features(5000, 17)
    yt = _teacher_labels(xt, 18)
    acc = np.mean((MF.infer(mem, p1, xt) > 0) == (yt > 0.5))
    assert acc > 0.85
    # the oracle's loss agrees that training helped
    assert M.loss_and_grad(p1, xt, yt, 1.0)[0] < M.loss_and_grad(p0, xt, yt, 1.0)[0]


def test_mlp_one_adam_step_matches_oracle(mem):
    x = _features(1024, 12)
    y = _teacher_labels(x, 13)
    p0 = M.init_params(14)
    p1, _ = MF.train(mem, p0, x, y, epochs=1, batch=1024, lr=1e-3, seed=1)
    _, g = M.loss_and_grad(p0, x, y, 1.0)  # one batch = the whole set, order irrelevant
    z = np.zeros(M.N_PARAMS, np.float32)
    pr, _, _ = M.adam_step(p0, z, z, g.astype(np.float32), 1, 1e-3)
    # Adam's first step moves each weight by ~lr * sign(g); tiny |g| may differ in sign
    big = np.abs(g) > 1e-3 * np.abs(g).max()
    assert np.allclose(p1[big], pr[big], atol=2e-5)


# ---- the filter inside clustering runs ---------------------------------------
def _run(mem, hg, obj=pg.OBJ_MOD, seed=3, ex_iters=0):
    wg = pg.weighted_graph(mem, hg.rowptr, hg.col, None if obj == pg.OBJ_MOD else hg.w, objective=obj)
    cd = pg.get_objective(mem, wg, obj, 1.0)
    labels, st = pg.run_clustering(mem, wg, cd, method=pg.METHOD_LEIDEN_PLUS, ex_iters=ex_iters, seed=seed)
    return wg, labels, st


def _run_method(mem, hg, method, ex_iters=0, seed=3):
    wg = pg.weighted_graph(mem, hg.rowptr, hg.col, None, objective=pg.OBJ_MOD)
    cd = pg.get_objective(mem, wg, pg.OBJ_MOD, 1.0)
    labels, st = pg.run_clustering(mem, wg, cd, method=method, ex_iters=ex_iters, seed=seed)
    return wg, labels, st


def _accept_all():
    p = np.zeros(M.N_PARAMS, np.float32)
    p[M.O_B3] = 100.0
    return p


def _reject_all():
    p = np.zeros(M.N_PARAMS, np.float32)
    p[M.O_B3] = -100.0
    return p


def test_logging_collects_labelled_samples(mem):
    hg = G.small_sbm()
    MF.log_start(mem, capacity=200000, sample_rate=1.0, seed=1)
    _, labels, st = _run(mem, hg)
    x, y, rows = MF.log_stop(mem, 200000)
    assert rows == len(x) > hg.n  # at least the first sweep's vertices
    assert set(np.unique(y)) <= {0.0, 1.0}
    assert 0 < y.sum() < len(y)
    assert np.all((x[:, 0] >= 0) & (x[:, 1] >= 0) & (x[:, 1] <= 1) & (np.abs(x[:, 2]) <= 4))
    assert set(np.unique(x[:, 3])) <= {0.0, 1.0}
    # logging does not change the clustering
    _, labels2, _ = _run(mem, hg)
    assert np.array_equal(labels, labels2)


def test_filter_accepting_everything_is_exact(mem):
    """An accept-all network sweeps like the plain method: one filtered pass
    plus the judge's one exact pass equals the oracle's pLeiden+ with
    ex_iters = 1 bit for bit (the judge's pass is pass 1 of the same seed
    sequence)."""
    hg = G.small_dcsbm()
    og = O.Graph(hg.rowptr, hg.col, hg.w, objective=pg.OBJ_WMOD)
    cd_o = O.ClusterData(og, pg.OBJ_WMOD, 1.0)
    lo, so = O.run_clustering(og, cd_o, method=pg.METHOD_LEIDEN_PLUS, ex_iters=1, seed=3)
    MF.enable(mem, _accept_all(), 0.0)
    MF.stats(mem, reset=True)
    try:
        _, lg, sg = _run(mem, hg, obj=pg.OBJ_WMOD)
        ev, sk = MF.stats(mem)
    finally:
        MF.disable(mem)
    assert ev > 0 and sk == 0
    assert sg["filtered_passes"] == 1 and sg["passes"] == sg["filtered_passes"] + sg["exact_passes"]
    # a second pass gains less than 0.001 here: no fallback
    assert sg["fell_back"] == 0 and sg["exact_passes"] == 1
    assert np.array_equal(lo, lg)
    assert so.objective == sg["objective"]


def test_judge_falls_back_when_the_filter_loses_modularity(mem):
    """A reject-all network leaves pLeiden one filtered pass made of strict
    local moves and exact finest-level moves: 0.11 below what exact passes
    reach on this SBM.  The judge's exact pass sees more than 0.001 of gain,
    falls back to exact passes until stable and reports it; the result is then
    at least the plain method's one-pass modularity less the tolerance."""
    hg = G.small_sbm()
    _, _, plain = _run_method(mem, hg, pg.METHOD_LEIDEN, ex_iters=0)
    assert plain["filtered_passes"] == 0 and plain["exact_passes"] == 0 and plain["fell_back"] == 0
    MF.enable(mem, _reject_all(), 0.0)
    try:
        wg, lg, sg = _run_method(mem, hg, pg.METHOD_LEIDEN, ex_iters=0)
    finally:
        MF.disable(mem)
    assert sg["filtered_passes"] == 1
    assert sg["fell_back"] == 1
    assert sg["judge_gain"] > 0.001
    assert sg["exact_passes"] >= 2
    q, _ = pg.verify_objective(mem, wg, lg, pg.OBJ_MOD)
    assert abs(q - sg["objective"]) < 1e-9
    assert sg["objective"] >= plain["objective"] - 0.001


def test_filter_rejecting_everything_still_yields_a_valid_clustering(mem):
    hg = G.small_sbm()
    MF.enable(mem, _reject_all(), 0.0)
    MF.stats(mem, reset=True)
    try:
        wg, lg, sg = _run(mem, hg)
        ev, sk = MF.stats(mem)
    finally:
        MF.disable(mem)
    assert ev == 0 and sk > 0
    assert lg.min() >= 0 and lg.max() < hg.n
    q, _ = pg.verify_objective(mem, wg, lg, pg.OBJ_MOD)
    assert abs(q - sg["objective"]) < 1e-9
    # the strict and the exact finest-level sweeps still find structure
    assert q > 0.1


def test_trained_filter_skips_work_at_equal_modularity(mem):
    """Train on logs of plain runs at seeds 1-4, evaluate on unseen seed 99."""
    xs, ys = [], []
    for s in (1, 2, 3, 4):
        hg = G.small_dcsbm(seed=s)
        MF.log_start(mem, capacity=400000, sample_rate=0.5, seed=s)
        _run(mem, hg, obj=pg.OBJ_WMOD, seed=s)
        x, y, _ = MF.log_stop(mem, 400000)
        xs.append(x)
        ys.append(y)
    x = np.concatenate(xs)
    y = np.concatenate(ys)
    pos_w = float((len(y) - y.sum()) / max(y.sum(), 1.0))
    p, losses = MF.train(mem, M.init_params(1), x, y, epochs=8, batch=2048, lr=3e-3, pos_weight=min(pos_w, 20.0))
    assert losses[-1] < losses[0]
    thr = MF.threshold_for_recall(mem, p, x, y, recall=0.98)
    hg = G.small_dcsbm(seed=99)
    t0 = time.perf_counter()
    _, _, plain = _run(mem, hg, obj=pg.OBJ_WMOD, seed=99, ex_iters=-1)
    t_plain = time.perf_counter() - t0
    MF.enable(mem, p, thr)
    MF.stats(mem, reset=True)
    try:
        t0 = time.perf_counter()
        _, _, learned = _run(mem, hg, obj=pg.OBJ_WMOD, seed=99, ex_iters=-1)
        t_learned = time.perf_counter() - t0
        ev, sk = MF.stats(mem)
    finally:
        MF.disable(mem)
    skipped = sk / max(ev + sk, 1)
    print(f"skipped {skipped:.3f} of filtered evaluations; Q plain {plain['objective']:.5f} "
          f"learned {learned['objective']:.5f}; passes {plain['passes']} vs {learned['filtered_passes']} filtered + "
          f"{learned['exact_passes']} exact; seconds {t_plain:.3f} vs {t_learned:.3f}")
    assert learned["filtered_passes"] >= 1 and learned["exact_passes"] >= 1
    assert skipped > 0.2
    # modularity within 0.001 of the plain method's (the judge's tolerance)
    assert learned["objective"] >= plain["objective"] - 0.001
