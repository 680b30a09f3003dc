"""CPU oracle for the learned move filter's network (TEST INFRASTRUCTURE ONLY).

Only tests and the benchmark's CPU leg may import this module; the product
path never does.  The reference has no learned filter (it is an addition of
this project), so this file restates the network's own definition:

  8 features -> 32 (ReLU) -> 32 (ReLU) -> 1 logit, BF16 weights, FP32
  accumulation.

Arithmetic, shared with the CUDA kernels:

* inputs and the weights of layers 1 and 2 are rounded to BF16 (round to
  nearest even) before the products; layer-1 activations are rounded to BF16
  before layer 2 (they feed a BF16 tensor-core product on the GPU);
* layer-2 activations stay FP32 and meet BF16-rounded layer-3 weights;
* biases are FP32;
* loss: positive-weighted binary cross-entropy on the logit, averaged over
  the batch; gradients flow straight through the BF16 roundings to the FP32
  master weights.

Parameter layout (one flat FP32 vector of N_PARAMS):
  W1[32][8] | b1[32] | W2[32][32] | b2[32] | W3[32] | b3
"""
import numpy as np

N_IN, N_H = 8, 32
O_W1, O_B1 = 0, 256
O_W2, O_B2 = 288, 1312
O_W3, O_B3 = 1344, 1376
N_PARAMS = 1377


def bf16(x):
    """Round float32 values to the nearest BF16 value (ties to even), as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    # NaN stays NaN
    return np.where(np.isnan(a), a, out).reshape(np.shape(x))


def unpack(p):
    p = np.asarray(p)
    if p.dtype != np.float64:
        p = p.astype(np.float32)
    return (p[O_W1:O_B1].reshape(N_H, N_IN), p[O_B1:O_W2], p[O_W2:O_B2].reshape(N_H, N_H), p[O_B2:O_W3],
            p[O_W3:O_B3], p[O_B3])


def init_params(seed):
    """He-style uniform init with a fixed generator (the GPU trainer uses the same values when given them)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    p[O_W1:O_B1] = rng.uniform(-1, 1, N_H * N_IN) * np.sqrt(6.0 / N_IN)
    p[O_W2:O_B2] = rng.uniform(-1, 1, N_H * N_H) * np.sqrt(6.0 / N_H)
    p[O_W3:O_B3] = rng.uniform(-1, 1, N_H) * np.sqrt(6.0 / N_H)
    return p.astype(np.float32)


def forward(p, x, rounding=True):
    """Returns (logit, cache) for features x [N, 8] (float32); computed in float64 from float32 inputs.

    rounding=False drops every BF16 rounding (a smooth network, used to check
    the backward pass against finite differences)."""
    W1, b1, W2, b2, W3, b3 = unpack(np.asarray(p, np.float32) if rounding else np.asarray(p, np.float64))
    if rounding:
        rnd = lambda a: bf16(np.asarray(a, np.float32)).astype(np.float64)  # noqa: E731
        f32 = lambda a: np.asarray(a, np.float32).astype(np.float64)  # noqa: E731
    else:
        rnd = f32 = lambda a: np.asarray(a, np.float64)  # noqa: E731
    xb = rnd(x)
    W1b, W2b, W3b = rnd(W1), rnd(W2), rnd(W3)
    z1 = xb @ W1b.T + b1.astype(np.float64)
    h1b = rnd(f32(np.maximum(z1, 0.0)))
    z2 = h1b @ W2b.T + b2.astype(np.float64)
    h2 = f32(np.maximum(z2, 0.0))
    logit = h2 @ W3b + np.float64(b3)
    return logit, (xb, z1, h1b, z2, h2, W2b, W3b)


def loss_and_grad(p, x, y, pos_weight, rounding=True):
    """Mean positive-weighted BCE and its gradient (float64) w.r.t. the flat parameters."""
    y = np.asarray(y, np.float64)
    logit, (xb, z1, h1b, z2, h2, W2b, W3b) = forward(p, x, rounding)
    n = len(y)
    sp = 1.0 / (1.0 + np.exp(-logit))
    # -[w y log s + (1-y) log(1-s)]
    log_s = -np.logaddexp(0.0, -logit)
    log_1s = -np.logaddexp(0.0, logit)
    loss = -(pos_weight * y * log_s + (1.0 - y) * log_1s).mean()
    dl = (pos_weight * y * (sp - 1.0) + (1.0 - y) * sp) / n
    g = np.zeros(N_PARAMS, np.float64)
    g[O_W3:O_B3] = dl @ h2
    g[O_B3] = dl.sum()
    dh2 = np.outer(dl, W3b) * (z2 > 0)
    g[O_W2:O_B2] = (dh2.T @ h1b).ravel()
    g[O_B2:O_W3] = dh2.sum(0)
    dh1 = (dh2 @ W2b) * (z1 > 0)
    g[O_W1:O_B1] = (dh1.T @ xb).ravel()
    g[O_B1:O_W2] = dh1.sum(0)
    return loss, g


def adam_step(p, m, v, g, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (float32 state), returning new (p, m, v)."""
    p = np.asarray(p, np.float32).copy()
    m = (b1 * m + (1 - b1) * g).astype(np.float32)
    v = (b2 * v + (1 - b2) * g * g).astype(np.float32)
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    p = (p - lr * mh / (np.sqrt(vh) + eps)).astype(np.float32)
    return p, m, v
