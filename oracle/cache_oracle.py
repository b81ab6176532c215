"""ORACLE -- test infrastructure only.  numpy FP64 restatement of the learned radiance cache
(stratum2_b200/csrc/s2_cache.cuh): the multiresolution hash-grid encoding (Instant-NGP, Mueller et
al. 2022) and the 32 -> 64 -> 64 -> 3 ReLU MLP without biases, with the device's f16 roundings of
parameters, encoded features and hidden activations, and the relative L2 loss with its gradients.
The radiance cache has no counterpart in the reference."""
from __future__ import annotations

import numpy as np

LEVELS, FEATURES, IN, HIDDEN, OUT = 16, 2, 32, 64, 3
W1, W2, W3 = HIDDEN * IN, HIDDEN * HIDDEN, OUT * HIDDEN


def f16(x):
    return np.asarray(x, np.float64).astype(np.float16).astype(np.float64)


def resolutions(base=16, top=2048, log2_table=19):
    b = np.exp((np.log(top) - np.log(base)) / (LEVELS - 1))
    res = np.floor(base * b ** np.arange(LEVELS) + 1e-9)
    dense = 8 * ((res.astype(np.int64) + 2) // 2) ** 3 <= 2 ** log2_table
    return res, dense


def corner_index(level, x, y, z, res, dense, log2_table):
    """Table entry of grid vertex (x, y, z): 2x2x2 bricks of 8 consecutive entries, placed densely
    or by the Instant-NGP spatial hash of the brick coordinates (s2_cache.cuh cache_index)."""
    mask = np.uint64((1 << (log2_table - 3)) - 1)
    x, y, z = (np.asarray(v, np.uint64) for v in (x, y, z))
    one = np.uint64(1)
    bx, by, bz = x >> one, y >> one, z >> one
    if dense[level]:
        n = np.uint64((int(res[level]) + 2) // 2)
        b = (bx + n * (by + n * bz)) & mask
    else:
        b = (bx ^ ((by * np.uint64(2654435761)) & np.uint64(0xFFFFFFFF)) ^
             ((bz * np.uint64(805459861)) & np.uint64(0xFFFFFFFF))) & mask
    return ((b << np.uint64(3)) | (x & one) | ((y & one) << one) | ((z & one) << np.uint64(2))).astype(np.int64)


def unit(pos, box_min, box_max):
    u = (np.asarray(pos, np.float64) - np.asarray(box_min, np.float64)) / (np.asarray(box_max, np.float64) - box_min)
    return np.clip(u, 0.0, 0.99999994)


def encode(pos, table, box_min, box_max, base=16, top=2048, with_corners=False):
    """Features (n, 32) in f64 before the f16 rounding; table (levels, T, 2) f64 (already f16-valued).
    with_corners also returns, per level, the corner indices (n, 8) and weights (n, 8)."""
    log2_table = int(np.log2(table.shape[1]))
    res, dense = resolutions(base, top, log2_table)
    u = unit(pos, box_min, box_max)
    n = u.shape[0]
    feats = np.zeros((n, IN))
    corners = []
    for l in range(LEVELS):
        f = u * res[l]
        i0 = np.floor(f)
        w = f - i0
        i0 = i0.astype(np.int64)
        idx = np.zeros((n, 8), np.int64)
        wt = np.zeros((n, 8))
        for k in range(8):
            d = np.array([k & 1, (k >> 1) & 1, k >> 2])
            wk = np.prod(np.where(d == 1, w, 1 - w), axis=1)
            ik = corner_index(l, i0[:, 0] + d[0], i0[:, 1] + d[1], i0[:, 2] + d[2], res, dense, log2_table)
            idx[:, k] = ik
            wt[:, k] = wk
            feats[:, 2 * l:2 * l + 2] += wk[:, None] * table[l, ik]
        corners.append((idx, wt))
    return (feats, corners) if with_corners else feats


def split(weights):
    w = np.asarray(weights, np.float64)
    return w[:W1].reshape(HIDDEN, IN), w[W1:W1 + W2].reshape(HIDDEN, HIDDEN), w[W1 + W2:].reshape(OUT, HIDDEN)


def forward(pos, weights, table, box_min, box_max, base=16, top=2048):
    """Cache output (n, 3) with the device's f16 roundings (f64 accumulation)."""
    a, b, c = (f16(m) for m in split(weights))
    x = f16(encode(pos, f16(table), box_min, box_max, base, top))
    h1 = f16(np.maximum(x @ a.T, 0))
    h2 = f16(np.maximum(h1 @ b.T, 0))
    return h2 @ c.T


def _r(x, exact):
    return np.asarray(x, np.float64) if exact else f16(x)


def loss_and_grads(pos, targets, weights, table, box_min, box_max, base=16, top=2048, exact=False,
                   grad_scale=1.0 / 64.0):
    """Mean relative L2 loss over the records (sum_c (y_c - t_c)^2 / (y_c^2 + 0.01) / 3 per record,
    denominator held constant) and its gradients with respect to the weights (6336) and the table
    (levels, T, 2).  exact=False applies the device's f16 roundings (parameters, features, hidden
    activations and the backward activations scaled by grad_scale); exact=True is plain f64 math."""
    n = len(pos)
    a, b, c = (_r(m, exact) for m in split(weights))
    tab = _r(table, exact)
    feats, corners = encode(pos, tab, box_min, box_max, base, top, with_corners=True)
    x = _r(feats, exact)
    h1 = _r(np.maximum(x @ a.T, 0), exact)
    h2 = _r(np.maximum(h1 @ b.T, 0), exact)
    y = h2 @ c.T
    t = np.asarray(targets, np.float64)[:, :3]
    d = y - t
    den = y * y + 0.01
    loss = float(np.mean(np.sum(d * d / den, 1) / 3))
    dy = 2 * d / den / 3
    if not exact:
        dy = np.clip(dy, -1e4, 1e4)
    s = 1.0 if exact else grad_scale
    dw3 = dy.T @ h2
    dh2 = _r((dy @ c) * (h2 > 0) * s, exact)
    dw2 = dh2.T @ h1 / s
    dh1 = _r((dh2 @ b) * (h1 > 0), exact)
    dw1 = dh1.T @ x / s
    dx = dh1 @ a / s
    gt = np.zeros_like(np.asarray(table, np.float64))
    for l, (idx, wt) in enumerate(corners):
        for k in range(8):
            np.add.at(gt[l, :, 0], idx[:, k], wt[:, k] * dx[:, 2 * l])
            np.add.at(gt[l, :, 1], idx[:, k], wt[:, k] * dx[:, 2 * l + 1])
    gw = np.concatenate([dw1.ravel(), dw2.ravel(), dw3.ravel()])
    return loss, gw / n, gt / n


def loss_only(pos, targets, weights, table, box_min, box_max, base=16, top=2048):
    """f64 loss with the denominator evaluated at the given parameters (for finite differences of
    loss_and_grads(exact=True), hold `den` by passing the same parameters)."""
    a, b, c = split(weights)
    x = encode(pos, np.asarray(table, np.float64), box_min, box_max, base, top)
    y = np.maximum(np.maximum(x @ a.T, 0) @ b.T, 0) @ c.T
    t = np.asarray(targets, np.float64)[:, :3]
    return y, t
