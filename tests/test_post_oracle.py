"""The numpy oracle of the post-processing passes (oracle/post_oracle.py): its colour helpers
pinned against the reference's own compat/common.h (compiled into oracle/_ref/libref_compat.so),
and closed-form properties of the accumulation and the operators.  CPU only."""
import ctypes as C
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle_lib import ref_compat

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import post_oracle as po  # noqa: E402

needs_ref = pytest.mark.skipif(ref_compat() is None, reason="reference compat probe not built (reference tree absent)")


@needs_ref
def test_colour_helpers_match_reference_compat_header():
    L = ref_compat()
    L.ref_luminance.restype = C.c_float
    rng = np.random.default_rng(0)
    for _ in range(300):
        rgb = rng.uniform(0, 2, 3).astype(np.float32)
        out = np.zeros(3, np.float32)
        L.ref_rgb_to_srgb(rgb.ctypes.data, out.ctypes.data)
        np.testing.assert_allclose(po.rgb_to_srgb_reference(rgb), out, rtol=2e-6, atol=1e-7)
        x = np.float32(rng.uniform(0, 1))
        L.ref_viridis(C.c_float(x), out.ctypes.data)
        # float32 evaluation of a quintic with coefficients up to 33 in the reference
        np.testing.assert_allclose(po.viridis(x), out, rtol=1e-5, atol=2e-5)
        assert abs(po.luminance(rgb) - L.ref_luminance(rgb.ctypes.data)) < 1e-6


def test_reference_gamma_is_not_srgb():
    # the reference's rgbToSrgb scales before the power: it differs from sRGB above 0.0031308
    x = np.array([0.001, 0.01, 0.2, 0.5, 1.0])
    assert np.allclose(po.rgb_to_srgb(x)[[0]], po.rgb_to_srgb_reference(x)[[0]])
    assert np.all(np.abs(po.rgb_to_srgb(x)[1:] - po.rgb_to_srgb_reference(x)[1:]) > 1e-3)
    assert abs(po.rgb_to_srgb(1.0) - 1.0) < 1e-12


def test_static_accumulation_is_the_running_mean():
    rng = np.random.default_rng(1)
    frames = [np.concatenate([rng.uniform(0, 1, (4, 5, 3)), np.ones((4, 5, 1))], -1) for _ in range(6)]
    prev = None
    for k, f in enumerate(frames):
        c, m = po.temporal_accumulate(f, None, None, None, None, prev, flags=0)
        prev = {"color": c, "moments": m}
        np.testing.assert_allclose(c[..., :3], np.mean(frames[:k + 1], 0)[..., :3], rtol=1e-12)
        np.testing.assert_allclose(c[..., 3], k + 1)
    # a history limit turns it into an exponential average with weight 1 / limit
    c, _ = po.temporal_accumulate(frames[0], None, None, None, None, {"color": c, "moments": m}, flags=0, history_limit=4)
    np.testing.assert_allclose(c[..., 3], 4)


def test_operators_closed_forms():
    c = np.full((1, 1, 4), 3.0)
    assert np.allclose(po.tonemap(c, 0)[..., :3], 3.0)                       # raw
    assert np.allclose(po.tonemap(c, 3)[..., :3], 0.75)                      # luminance Reinhard: 3 / 4
    assert np.allclose(po.tonemap(c, 0, exposure=1.0)[..., :3], 6.0)         # 2^exposure
    assert np.allclose(po.tonemap(c, 2)[..., :3], 3 / 4 * (1 + 3 / 9))       # extended with max 3
    assert np.all(po.tonemap(c, 8)[..., :3] <= 1)                            # ACES approximation saturates
