"""Batched streaming renders (s2_render_views): many views per call, path regeneration, CUDA-graph
replay and fixed-point accumulation, checked against the per-view wave renderer (s2_render)."""
import numpy as np
import pytest

from stratum2_b200 import _abi
from stratum2_b200.scene import look_at_rotation, make_view
from stratum2_b200.scenegen import box_scene, terrain_scene

pytestmark = pytest.mark.gpu
J = _abi.FLAG_PIXEL_JITTER


def params(spp, flags, seed=3, wave=0, minl=2, maxl=5):
    p = _abi.S2RenderParams()
    _abi.lib().s2_default_render_params(p)
    p.spp, p.flags, p.frame_seed, p.wave_paths = spp, flags, seed, wave
    p.min_path_length, p.max_path_length = minl, maxl
    return p


@pytest.fixture(scope="module")
def box(device):
    wl = box_scene(seed=1, width=64, height=64)
    device.upload_scene(wl.scene)
    views = [wl.view,
             make_view((0.3, -0.2, 2.5), 48, 32, 50.0, look_at_rotation((0.3, -0.2, 2.5), (0, 0, 0))),
             make_view((-0.5, 0.4, 2.8), 17, 23, 35.0, look_at_rotation((-0.5, 0.4, 2.8), (0.1, 0, 0)))]
    return wl, views


def test_views_match_per_view_renders(device, box):
    wl, views = box
    device.upload_scene(wl.scene)
    p = params(16, _abi.FLAG_LAMBERTIAN | J)
    res, st = device.render_views(views, p)
    total = 0
    for v, r in zip(views, res):
        w, h = v.image_max[0], v.image_max[1]
        ref = device.render(v, w, h, params=params(16, _abi.FLAG_LAMBERTIAN | J))
        np.testing.assert_allclose(r.radiance, ref.radiance, rtol=1e-5, atol=1e-6)
        np.testing.assert_array_equal(r.albedo, ref.albedo)
        np.testing.assert_array_equal(r.visibility, ref.visibility)
        np.testing.assert_array_equal(r.ids32, ref.ids32)
        np.testing.assert_allclose(r.depth, ref.depth, rtol=1e-6)
        total += w * h * 16
    assert st.paths == total and st.extension_rays > 0


def test_deterministic_regeneration_and_progressive(device, box):
    wl, views = box
    device.upload_scene(wl.scene)
    base, _ = device.render_views(views, params(16, _abi.FLAG_LAMBERTIAN | J))
    again, _ = device.render_views(views, params(16, _abi.FLAG_LAMBERTIAN | J))
    small, st_small = device.render_views(views, params(16, _abi.FLAG_LAMBERTIAN | J, wave=4096))
    device.render_views(views, params(8, _abi.FLAG_LAMBERTIAN | J, seed=3))
    prog, _ = device.render_views(views, params(8, _abi.FLAG_LAMBERTIAN | J | _abi.FLAG_ACCUMULATE, seed=11))
    assert st_small.kernel_launches > 100  # the small queue replays the bounce graph many times
    for a, b, c, d in zip(base, again, small, prog):
        np.testing.assert_array_equal(a.radiance, b.radiance)   # integer sums: bit-identical
        np.testing.assert_array_equal(a.radiance, c.radiance)   # independent of the queue size
        np.testing.assert_array_equal(a.radiance, d.radiance)   # 8 + 8 spp == 16 spp


def test_sixteen_views_terrain(device):
    wl = terrain_scene(seed=2, grid=128, spheres=8, sphere_level=2, width=64, height=36, tiles=2, area_lights=2,
                       sun_radiance=50.0, sun_cone_degrees=5.0)
    device.upload_scene(wl.scene)
    rng = np.random.default_rng(4)
    views = []
    for k in range(16):
        w = int(np.exp(rng.uniform(np.log(16), np.log(96))))
        h = int(np.exp(rng.uniform(np.log(16), np.log(64))))
        pos = (rng.uniform(-0.8, 0.8), rng.uniform(0.5, 1.2), rng.uniform(1.2, 2.0))
        views.append(make_view(pos, w, h, 45.0, look_at_rotation(pos, (0, 0, 0))))
    res, st = device.render_views(views, params(4, J, minl=1, maxl=6))
    assert st.paths == sum((v.image_max[0] * v.image_max[1]) * 4 for v in views)
    for v, r in zip(views, res):
        ref = device.render(v, v.image_max[0], v.image_max[1], params=params(4, J, minl=1, maxl=6))
        np.testing.assert_allclose(r.radiance, ref.radiance, rtol=1e-5, atol=1e-5)
