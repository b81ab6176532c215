"""Image metrics against the reference's ImageComparer (src/Shaders/kernels/image_compare.slang:27-36,
normalised in src/App/ImageComparer.cpp:180-186): per pixel the RGB error summed with dot(1, e3),
summed over the image, divided by 3*W*H; the MSE mode is reported as its square root.

Two deliberate differences, both where the reference's result is not defined or not exact:
* SMAPE of a channel that is 0 in both images is 0/0.  In the shader the NaN enters the wave's
  WaveActiveSum and the `(uint)` conversion of a NaN is undefined (it zeroes the whole wave's sum
  on GPUs that convert NaN to 0); here such a channel contributes 0 and the others count.
* The shader accumulates wave sums as integers scaled by mQuantization (truncating each); here the
  sums are exact floating point."""
import numpy as np
import pytest

from stratum2_b200 import metrics


def _reference_semantics(a, b, mode):
    """The shader's arithmetic per pixel in float64, before its quantization."""
    c1, c2 = a[..., :3].astype(np.float64), b[..., :3].astype(np.float64)
    dc = np.abs(c1 - c2)
    if mode == "smape":
        with np.errstate(invalid="ignore", divide="ignore"):
            e3 = dc / (np.abs(c1) + np.abs(c2))
        e3 = np.where(np.isnan(e3), 0.0, e3)  # the per-channel 0/0 case, see the module docstring
    elif mode == "mse":
        e3 = dc ** 2
    else:
        e3 = dc
    total = e3.sum(-1).sum() / (3 * a.shape[0] * a.shape[1])
    return float(np.sqrt(total)) if mode == "mse" else float(total)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_metrics_follow_the_image_comparer(seed):
    rng = np.random.default_rng(seed)
    a = rng.uniform(0, 2, (17, 23, 4)).astype(np.float32)
    b = rng.uniform(0, 2, (17, 23, 4)).astype(np.float32)
    a[:3, :5, :3] = 0
    b[:3, :5, :3] = 0  # channels that are zero in both images
    b[5, 5, 1] = -0.5  # negative values enter |c| in the SMAPE denominator
    assert metrics.smape(a, b) == pytest.approx(_reference_semantics(a, b, "smape"), rel=1e-12)
    assert metrics.rmse(a, b) == pytest.approx(_reference_semantics(a, b, "mse"), rel=1e-12)
    assert metrics.mean_abs_error(a, b) == pytest.approx(_reference_semantics(a, b, "mae"), rel=1e-12)


def test_metrics_ignore_alpha_and_vanish_on_equal_images():
    rng = np.random.default_rng(7)
    a = rng.uniform(0, 1, (8, 8, 4))
    b = a.copy()
    b[..., 3] = 0.0
    assert metrics.smape(a, b) == 0.0 and metrics.rmse(a, b) == 0.0 and metrics.mean_abs_error(a, b) == 0.0
    assert metrics.relmse(a, b) == 0.0


def test_relmse_definition():
    a = np.full((2, 2, 3), 1.5)
    b = np.full((2, 2, 3), 1.0)
    assert metrics.relmse(a, b) == pytest.approx(0.25 / (1.0 + 1e-2))
