"""The radiance-cache oracle's analytic gradients (oracle/cache_oracle.py, exact f64 mode) agree
with central finite differences of its loss (the denominator y^2 + 0.01 held at the base point,
as the loss defines it).  CPU only."""
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import cache_oracle as co  # noqa: E402

BOX_MIN, BOX_MAX = np.array([-1.0, -1.0, -1.0]), np.array([1.0, 1.0, 1.0])


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    log2 = 10
    w = rng.normal(0, 0.3, co.W1 + co.W2 + co.W3)
    t = rng.uniform(-0.5, 0.5, (co.LEVELS, 1 << log2, 2))
    pos = rng.uniform(-1, 1, (16, 3))
    tgt = rng.uniform(0, 2, (16, 3))
    _, gw, gt = co.loss_and_grads(pos, tgt, w, t, BOX_MIN, BOX_MAX, exact=True)
    y0, tt = co.loss_only(pos, tgt, w, t, BOX_MIN, BOX_MAX)
    den = y0 * y0 + 0.01

    def loss(wv, tv):
        y, _ = co.loss_only(pos, tgt, wv, tv, BOX_MIN, BOX_MAX)
        return np.mean(np.sum((y - tt) ** 2 / den, 1) / 3)

    eps = 1e-6
    for i in rng.choice(len(w), 40, replace=False):
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        fd = (loss(wp, t) - loss(wm, t)) / (2 * eps)
        assert abs(fd - gw[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, gw[i])
    nz = np.argwhere(np.abs(gt) > 0)
    for l, e, f in nz[rng.choice(len(nz), 40, replace=False)]:
        tp, tm = t.copy(), t.copy()
        tp[l, e, f] += eps
        tm[l, e, f] -= eps
        fd = (loss(w, tp) - loss(w, tm)) / (2 * eps)
        assert abs(fd - gt[l, e, f]) <= 1e-6 + 1e-4 * abs(fd), (l, e, f, fd, gt[l, e, f])
