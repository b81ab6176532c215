"""Light tracing (S2_FLAG_LIGHT_TRACE, TestRenderer's mLightTrace mode: light subpaths connected to
the camera at every non-singular vertex, testrenderer.slang:441-512, 983-1020) estimates the same
image as path tracing: on the box scene it converges to the FP64 path-traced golden image (paths of
2..5 segments, jittered pixels = the box pixel filter the camera connections integrate over),
by the z-test of the other convergence tests.  Camera connections land in fixed-point pixel
totals, so renders are reproducible."""
from pathlib import Path

import numpy as np
import pytest

from stratum2_b200 import _abi
from stratum2_b200.scenegen import box_scene

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
LT = _abi.FLAG_LIGHT_TRACE | _abi.FLAG_LAMBERTIAN | _abi.FLAG_PIXEL_JITTER


def params(seed, spp, subpaths=1.0, flags=LT):
    p = _abi.S2RenderParams()
    _abi.lib().s2_default_render_params(p)
    p.spp, p.min_path_length, p.max_path_length, p.flags, p.frame_seed = spp, 2, 5, flags, seed
    p.light_subpaths = subpaths
    return p


def test_light_tracing_converges_to_path_traced_golden(device):
    wl = box_scene(seed=1, width=64, height=64)
    device.upload_scene(wl.scene)
    gold = np.load(GOLDEN / "box_64x64_fp64_16384spp.npz")
    means = np.stack([device.render(wl.view, 64, 64, params=params(1000 + 512 * b, 512, 2.0)).radiance[..., :3]
                      .astype(np.float64) for b in range(16)])
    m, v = means.mean(0), means.var(0, ddof=1) / 16
    ref, ref_v = gold["mean"], gold["var_of_mean"]
    z = (m - ref) / np.sqrt(v + ref_v + (1e-5 * np.abs(ref) + 1e-9) ** 2)
    assert np.mean(np.abs(z) > 5) <= 2e-3, f"{np.mean(np.abs(z) > 5):.4%} of pixel channels with |z| > 5"
    assert abs(z.mean()) < 0.15, z.mean()
    rel = (m.sum() - ref.sum()) / ref.sum()
    assert abs(rel) < 5e-3, rel


def test_light_tracing_is_reproducible_and_checks_arguments(device):
    wl = box_scene(seed=1, width=32, height=32)
    device.upload_scene(wl.scene)
    a = device.render(wl.view, 32, 32, params=params(5, 4))
    b = device.render(wl.view, 32, 32, params=params(5, 4))
    np.testing.assert_array_equal(a.radiance, b.radiance)
    assert a.stats.extension_rays > 0 and a.stats.shadow_rays > 0
    p = params(5, 4, flags=LT | _abi.FLAG_RESTIR_DI)
    with pytest.raises(_abi.S2Error) as e:
        device.render(wl.view, 32, 32, params=p)
    assert e.value.code == _abi.S2_ERR_UNSUPPORTED


def test_light_tracing_environment_and_emitters_match_path_tracing(device):
    """Sky with a 5-degree sun plus 64 emissive triangles over a terrain (Lambertian): light
    subpaths from the environment (parallel rays through a disc of the scene's bounding sphere,
    weighted by its area) and from the triangles converge to path tracing's image."""
    from stratum2_b200.scenegen import terrain_scene
    wl = terrain_scene(seed=2, grid=64, spheres=4, sphere_level=2, width=48, height=27, tiles=2, emissive_triangles=64,
                       emissive_sigma=0.5, emissive_power=0.02, emissive_height=(0.3, 0.6), emissive_edge=(0.02, 0.05),
                       sun_radiance=50.0, sun_cone_degrees=5.0, sky_scale=0.05)
    device.upload_scene(wl.scene)
    pt = params(0, 4096, flags=_abi.FLAG_LAMBERTIAN | _abi.FLAG_PIXEL_JITTER)
    ref = []
    for b in range(16):
        pt.frame_seed = 500000 + 4096 * b
        ref.append(device.render(wl.view, 48, 27, params=pt).radiance[..., :3].astype(np.float64))
    ref = np.stack(ref)
    lt = np.stack([device.render(wl.view, 48, 27, params=params(9000 + 1024 * b, 1024, 2.0)).radiance[..., :3]
                   .astype(np.float64) for b in range(16)])
    m, v = lt.mean(0), lt.var(0, ddof=1) / 16
    r, rv = ref.mean(0), ref.var(0, ddof=1) / 16
    z = (m - r) / np.sqrt(v + rv + (1e-5 * np.abs(r) + 1e-9) ** 2)
    assert np.mean(np.abs(z) > 5) <= 2e-3, f"{np.mean(np.abs(z) > 5):.4%} of pixel channels with |z| > 5"
    assert abs(z.mean()) < 0.15, z.mean()
    assert abs((m.sum() - r.sum()) / r.sum()) < 1e-2
