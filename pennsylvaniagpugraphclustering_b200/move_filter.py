"""The learned move filter: a small network that decides which vertices a
local-move sweep evaluates (gains of evaluated vertices stay exact).

This is a project addition with no counterpart in the reference.  The
workflow: log (features, moved) samples from plain runs
(:func:`log_start` / :func:`log_stop`), train the network on the GPU
(:func:`train`), pick a logit threshold that keeps almost every mover
(:func:`threshold_for_recall`), then :func:`enable` it on a context; every
``leiden_part`` / ``louvain_part`` / ``run_clustering`` on that context is then
filtered, except the finest level's last local move of each pass, which stays
exact.

Network: 8 features -> 32 -> 32 (ReLU) -> 1 logit, BF16 weights with FP32
accumulation; parameters are a flat float32 vector of :data:`N_PARAMS`
values (W1[32][8] | b1[32] | W2[32][32] | b2[32] | W3[32] | b3).  All calls go
through the C ABI (``pggc_mlp_*``, ``pggc_filter_*``).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from ._lib import MEM_HOST, check

N_PARAMS = 1377
N_FEATURES = 8


def _f32(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


def init_params(seed: int = 0) -> np.ndarray:
    """He-style uniform initial parameters (float32) from a seeded generator."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    p[0:256] = rng.uniform(-1, 1, 256) * np.sqrt(6.0 / 8)
    p[288:1312] = rng.uniform(-1, 1, 1024) * np.sqrt(6.0 / 32)
    p[1344:1376] = rng.uniform(-1, 1, 32) * np.sqrt(6.0 / 32)
    return p


def infer(mem, params, features) -> np.ndarray:
    """Logits of feature rows [N, 8] (tensor-core path)."""
    p = _f32(params, N_PARAMS)
    x = _f32(features).reshape(-1, N_FEATURES)
    out = np.empty(len(x), np.float32)
    check(L.lib().pggc_mlp_infer(mem.handle, p.ctypes.data, x.ctypes.data, len(x), MEM_HOST, out.ctypes.data))
    return out


def loss_grad(mem, params, features, labels, pos_weight: float = 1.0):
    """(mean positive-weighted BCE, gradient [N_PARAMS]) of one batch."""
    p = _f32(params, N_PARAMS)
    x = _f32(features).reshape(-1, N_FEATURES)
    y = _f32(labels, len(x))
    g = np.empty(N_PARAMS, np.float32)
    loss = np.empty(1, np.float32)
    check(L.lib().pggc_mlp_loss_grad(mem.handle, p.ctypes.data, x.ctypes.data, y.ctypes.data, len(x),
                                     float(pos_weight), MEM_HOST, g.ctypes.data, loss.ctypes.data))
    return float(loss[0]), g


def train(mem, params, features, labels, epochs=4, batch=4096, lr=3e-3, pos_weight=1.0, seed=1):
    """Adam training on the GPU; returns (new params, per-epoch mean loss)."""
    p = _f32(params, N_PARAMS).copy()
    x = _f32(features).reshape(-1, N_FEATURES)
    y = _f32(labels, len(x))
    losses = np.zeros(max(epochs, 1), np.float32)
    check(L.lib().pggc_mlp_train(mem.handle, p.ctypes.data, x.ctypes.data, y.ctypes.data, len(x), MEM_HOST,
                                 int(epochs), int(batch), float(lr), float(pos_weight), int(seed),
                                 losses.ctypes.data))
    return p, losses[:epochs]


def log_start(mem, capacity: int, sample_rate: float = 1.0, seed: int = 1):
    """Start logging (features, moved) samples from the context's plain sweeps."""
    check(L.lib().pggc_filter_log_start(mem.handle, int(capacity), float(sample_rate), int(seed)))


def log_label(mem, label: str = "moved"):
    """What logged samples are labelled with: "moved" (the vertex moves in the
    sweep) or "candidate" (the select step proposes a move for it)."""
    check(L.lib().pggc_filter_log_label(mem.handle, {"moved": 0, "candidate": 1}[label]))


def log_stop(mem, capacity: int):
    """Stop logging; returns (features [k, 8], labels [k], rows logged)."""
    x = np.empty((capacity, N_FEATURES), np.float32)
    y = np.empty(capacity, np.float32)
    cnt = ctypes.c_int64()
    check(L.lib().pggc_filter_log_stop(mem.handle, x.ctypes.data, y.ctypes.data, int(capacity), MEM_HOST,
                                       ctypes.byref(cnt)))
    k = min(cnt.value, capacity)
    return x[:k], y[:k], cnt.value


def threshold_for_recall(mem, params, features, labels, recall: float = 0.99) -> float:
    """The largest logit threshold that keeps `recall` of the positive rows."""
    lg = infer(mem, params, features)
    pos = np.sort(lg[np.asarray(labels) > 0.5])
    if len(pos) == 0:
        return float("-inf")
    k = int(np.floor((1.0 - recall) * len(pos)))
    return float(np.nextafter(pos[k], -np.inf))


def enable(mem, params, threshold: float):
    """Filter the context's sweeps with this network."""
    p = _f32(params, N_PARAMS)
    check(L.lib().pggc_filter_enable(mem.handle, p.ctypes.data, float(threshold)))


def disable(mem):
    check(L.lib().pggc_filter_enable(mem.handle, None, 0.0))


def scope(mem, max_pass: int = -1, min_level: int = 0):
    """Restrict the filter to passes before max_pass (< 0: all) and levels at
    or above min_level."""
    check(L.lib().pggc_filter_scope(mem.handle, int(max_pass), int(min_level)))


def stats(mem, reset: bool = False):
    """(vertices evaluated, vertices skipped) by the filter."""
    e, s = ctypes.c_int64(), ctypes.c_int64()
    check(L.lib().pggc_filter_stats(mem.handle, ctypes.byref(e), ctypes.byref(s), 1 if reset else 0))
    return e.value, s.value
