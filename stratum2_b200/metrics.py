"""Image comparison metrics.

`smape`, `rmse` and `mean_abs_error` restate the reference's ImageComparer
(src/Shaders/kernels/image_compare.slang:27-36, normalised in src/App/ImageComparer.cpp:180-186:
the per-channel error summed over RGB and pixels, divided by 3*W*H; MSE reported as its square
root).  `relmse` is the relative mean squared error used for convergence targets:
mean over pixels and RGB of (a - b)^2 / (b^2 + eps).

Differences from the shader, where its result is undefined or inexact: a SMAPE channel that is 0
in both images (0/0) contributes 0 here, where the shader's NaN makes the `(uint)` conversion of
its whole wave's sum undefined; and the sums are exact floating point, where the shader adds
wave sums truncated to integers after scaling by mQuantization.
"""
from __future__ import annotations

import numpy as np


def _rgb(x) -> np.ndarray:
    x = np.asarray(x, np.float64)
    return x[..., :3]


def smape(a, b) -> float:
    a, b = _rgb(a), _rgb(b)
    den = np.abs(a) + np.abs(b)
    e = np.where(den > 0, np.abs(a - b) / np.where(den > 0, den, 1), 0.0)
    return float(e.sum() / e.size)


def rmse(a, b) -> float:
    a, b = _rgb(a), _rgb(b)
    return float(np.sqrt(((a - b) ** 2).sum() / a.size))


def mean_abs_error(a, b) -> float:
    a, b = _rgb(a), _rgb(b)
    return float(np.abs(a - b).sum() / a.size)


def relmse(a, b, eps: float = 1e-2) -> float:
    """Relative MSE of `a` against reference `b`."""
    a, b = _rgb(a), _rgb(b)
    return float(np.mean((a - b) ** 2 / (b ** 2 + eps)))


def z_scores(a, b, var_a, var_b) -> np.ndarray:
    """Per-pixel, per-channel z statistic of two independent estimator means."""
    a, b = _rgb(a), _rgb(b)
    return (a - b) / np.sqrt(np.maximum(_rgb(var_a) + _rgb(var_b), 1e-30))
