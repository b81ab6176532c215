"""Learned radiance cache on the GPU (tcgen05 MLP over the hash-grid encoding) against the numpy
FP64 oracle (oracle/cache_oracle.py), which applies the same f16 roundings."""
import sys
from pathlib import Path

import numpy as np
import pytest

from stratum2_b200 import _abi

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import cache_oracle as co  # noqa: E402

pytestmark = pytest.mark.gpu
BOX_MIN, BOX_MAX = np.array([-1.0, -0.5, -2.0]), np.array([1.0, 1.5, 0.5])


def cache_params(log2_table=14, seed=3):
    p = _abi.S2CacheParams()
    _abi.lib().s2_cache_default_params(p)
    p.log2_table = log2_table
    p.seed = seed
    for k in range(3):
        p.box_min[k], p.box_max[k] = BOX_MIN[k], BOX_MAX[k]
    return p


def random_params(rng, log2_table):
    w = np.concatenate([rng.normal(0, np.sqrt(2 / co.IN), co.W1), rng.normal(0, np.sqrt(2 / co.HIDDEN), co.W2),
                        rng.normal(0, np.sqrt(1 / co.HIDDEN), co.W3)]).astype(np.float32)
    t = rng.uniform(-1, 1, (co.LEVELS, 1 << log2_table, 2)).astype(np.float32)
    return w, t


@pytest.mark.parametrize("n", [1, 127, 128, 1000, 20037])
def test_cache_query_matches_oracle(device, n):
    log2 = 14
    device.cache_init(cache_params(log2))
    rng = np.random.default_rng(n)
    w, t = random_params(rng, log2)
    device.cache_set_params(w, t)
    pos = rng.uniform(BOX_MIN - 0.1, BOX_MAX + 0.1, (n, 3))  # includes points clamped to the box
    g = device.cache_query(pos)
    o = co.forward(pos, w, t, BOX_MIN, BOX_MAX)
    scale = np.abs(o).max() + 1e-3
    err = np.abs(g - o) / scale
    assert err.max() < 2e-2, err.max()
    assert np.mean(err) < 2e-3, np.mean(err)


def test_cache_params_round_trip_and_init(device):
    device.cache_init(cache_params(12, seed=9))
    w0, t0 = device.cache_get_params()
    assert np.abs(t0).max() <= 1e-4 and np.abs(t0).max() > 0
    assert np.abs(w0[:co.W1]).max() <= np.sqrt(6 / (co.IN + co.HIDDEN)) + 1e-6
    rng = np.random.default_rng(1)
    w, t = random_params(rng, 12)
    device.cache_set_params(w, t)
    w1, t1 = device.cache_get_params()
    np.testing.assert_array_equal(w1, w)
    np.testing.assert_array_equal(t1, t)
    # default 2^19 table, box from the scene bounds needs a scene; an explicit box works without one
    device.cache_init(cache_params(19))
    g = device.cache_query(np.zeros((3, 3)))
    assert np.isfinite(g).all()


@pytest.mark.parametrize("n", [128, 1000, 4099])
def test_cache_gradients_match_oracle(device, n):
    log2 = 12
    device.cache_init(cache_params(log2))
    rng = np.random.default_rng(10 + n)
    w, t = random_params(rng, log2)
    t *= 0.3
    device.cache_set_params(w, t)
    pos = rng.uniform(BOX_MIN, BOX_MAX, (n, 3))
    tgt = rng.uniform(0, 2, (n, 3))
    loss, gw, gt = device.cache_gradients(pos, tgt)
    oloss, ow, ot = co.loss_and_grads(pos, tgt, w, t, BOX_MIN, BOX_MAX)
    assert abs(loss - oloss) <= 1e-3 * abs(oloss) + 1e-6, (loss, oloss)
    for name, g, o in (("W1", gw[:co.W1], ow[:co.W1]), ("W2", gw[co.W1:co.W1 + co.W2], ow[co.W1:co.W1 + co.W2]),
                       ("W3", gw[co.W1 + co.W2:], ow[co.W1 + co.W2:]), ("table", gt.ravel(), ot.ravel())):
        rel = np.linalg.norm(g - o) / (np.linalg.norm(o) + 1e-12)
        assert rel < 2e-2, f"{name}: relative gradient error {rel:.4f}"


def test_cache_training_fits_a_smooth_field(device):
    """Online training on a smooth radiance field: the loss falls and held-out predictions follow it."""
    device.cache_init(cache_params(16))
    rng = np.random.default_rng(5)

    def field(p):
        return np.stack([1 + 0.5 * np.sin(3 * p[:, 0]), 1 + 0.5 * np.cos(2 * p[:, 1] + p[:, 2]),
                         0.5 + 0.25 * np.sin(p[:, 0] * p[:, 2] * 4)], 1)

    losses = []
    for step in range(300):
        pos = rng.uniform(BOX_MIN, BOX_MAX, (1 << 14, 3))
        losses.append(device.cache_train(pos, field(pos)))
    test = rng.uniform(BOX_MIN, BOX_MAX, (4096, 3))
    pred = device.cache_query(test)
    ref = field(test)
    rel = np.mean((pred - ref) ** 2 / (ref ** 2 + 1e-2))
    assert np.mean(losses[-10:]) < 0.05 * np.mean(losses[:3]), (losses[:3], losses[-10:])
    assert rel < 5e-3, rel
