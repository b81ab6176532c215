"""The radiance cache inside the path tracer (S2_FLAG_RADIANCE_CACHE): with the cache beyond the
maximum path length the render is the plain render (training paths are plain paths and training
does not touch the image; the shade kernel's cache instantiation may round a few contributions
differently, so the comparison allows 1e-5 relative); with paths ending in the cache, the
progressive image after online training stays close to the FP64 golden image while its per-frame
noise is lower than the plain path tracer's.  Both also through the batched entry point
(s2_render_views), whose training paths are extra paths with their own accumulators."""
from pathlib import Path

import numpy as np
import pytest

from stratum2_b200 import _abi
from stratum2_b200.metrics import relmse
from test_render_gpu import make_params, terrain_wl

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
J = _abi.FLAG_PIXEL_JITTER
CACHE = _abi.FLAG_RADIANCE_CACHE


@pytest.fixture(scope="module")
def terrain(device):
    wl = terrain_wl()
    device.upload_scene(wl.scene)
    device.cache_init()
    return wl


def test_cache_beyond_max_length_is_the_plain_render(device, terrain):
    wl = terrain
    device.upload_scene(wl.scene)
    device.cache_init()
    p = make_params(4, 1, 6, J, seed=21)
    plain = device.render(wl.view, wl.width, wl.height, params=p)
    p.flags |= CACHE
    p.cache_bounces = 10
    p.cache_train_paths = 512
    cached = device.render(wl.view, wl.width, wl.height, params=p)
    # the same estimator in another instantiation of the shade kernel: its floating-point
    # contractions and approximate quotients may round differently in the last bits
    np.testing.assert_allclose(cached.radiance, plain.radiance, rtol=1e-4, atol=1e-7)
    w_after, _ = device.cache_get_params()
    device.cache_init()
    w0, _ = device.cache_get_params()
    assert not np.array_equal(w_after, w0)  # the render trained the cache


def test_cached_render_close_to_golden_with_less_noise(device, terrain):
    wl = terrain
    device.upload_scene(wl.scene)
    device.cache_init()
    gold = np.load(GOLDEN / "terrain_64x36_fp64_131072spp.npz")
    ref = gold["mean"].astype(np.float64)
    p = make_params(1, 1, 6, J | CACHE)
    p.cache_train_paths = 1024
    frames = []
    for f in range(1024):
        p.frame_seed = 7000 + f
        frames.append(device.render(wl.view, wl.width, wl.height, params=p).radiance[..., :3].astype(np.float64))
    frames = np.stack(frames)
    late = frames[512:]
    plain = np.stack([device.render(wl.view, wl.width, wl.height, params=make_params(1, 1, 6, J, seed=90000 + f))
                      .radiance[..., :3].astype(np.float64) for f in range(512)])
    err_cache = relmse(late.mean(0), ref)
    var_cache = np.mean(late.var(0) / (ref ** 2 + 1e-2))
    var_plain = np.mean(plain.var(0) / (ref ** 2 + 1e-2))
    print("cache relMSE", err_cache, "per-frame relvar cache", var_cache, "plain", var_plain)
    assert err_cache < 0.02, err_cache
    assert var_cache < var_plain, (var_cache, var_plain)


def test_batched_cache_beyond_max_length_is_the_batched_render_and_trains(device, terrain):
    """Batched streaming entry point: training paths are extra paths with their own accumulators,
    so with the cache beyond the maximum path length the image is the batched render (up to the
    cache shade instantiation's rounding, 1e-5 relative measured), and the call still trains the
    cache."""
    wl = terrain
    device.upload_scene(wl.scene)
    device.cache_init()
    w0, _ = device.cache_get_params()
    p = make_params(4, 1, 6, J, seed=21)
    plain, _ = device.render_views([wl.view], p)
    p.flags |= CACHE
    p.cache_bounces = 10
    p.cache_train_paths = 512
    cached, _ = device.render_views([wl.view], p)
    np.testing.assert_allclose(cached[0].radiance, plain[0].radiance, rtol=3e-5, atol=1e-7)
    w1, _ = device.cache_get_params()
    assert not np.array_equal(w1, w0)


def test_batched_cached_render_close_to_golden_with_less_noise(device, terrain):
    """The batched + radiance-cache form: progressive 1-spp calls of s2_render_views (accumulated on
    the device) with online training stay close to the FP64 golden image, with lower per-frame
    noise than plain batched path tracing."""
    wl = terrain
    device.upload_scene(wl.scene)
    device.cache_init()
    gold = np.load(GOLDEN / "terrain_64x36_fp64_131072spp.npz")
    ref = gold["mean"].astype(np.float64)
    p = make_params(1, 1, 6, J | CACHE)
    p.cache_train_paths = 1024
    frames = []
    for f in range(1024):
        p.frame_seed = 7000 + f
        r, _ = device.render_views([wl.view], p)
        frames.append(r[0].radiance[..., :3].astype(np.float64))
    late = np.stack(frames[512:])
    plain = []
    for f in range(512):
        r, _ = device.render_views([wl.view], make_params(1, 1, 6, J, seed=90000 + f))
        plain.append(r[0].radiance[..., :3].astype(np.float64))
    plain = np.stack(plain)
    err_cache = relmse(late.mean(0), ref)
    var_cache = np.mean(late.var(0) / (ref ** 2 + 1e-2))
    var_plain = np.mean(plain.var(0) / (ref ** 2 + 1e-2))
    print("batched cache relMSE", err_cache, "per-frame relvar cache", var_cache, "plain", var_plain)
    assert err_cache < 0.02, err_cache
    assert var_cache < var_plain, (var_cache, var_plain)
