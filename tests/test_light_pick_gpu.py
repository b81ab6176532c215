"""Power-proportional light selection (S2_FLAG_LIGHT_POWER_PICK; the reference picks lights
uniformly, lights.hlsli:200, which stays the default).  The pick changes only the distribution of
the light samples, so plain NEE and RIS must converge to the uniform-pick image; on a scene of 256
emitters with lognormal(0, 1) power it must lower the per-frame error."""
import numpy as np
import pytest
import torch

from stratum2_b200 import _abi
from stratum2_b200.scenegen import terrain_scene

pytestmark = pytest.mark.gpu
J = _abi.FLAG_PIXEL_JITTER | _abi.FLAG_LAMBERTIAN
POWER = _abi.FLAG_LIGHT_POWER_PICK


def params(seed, flags, spp=1, m=4):
    p = _abi.S2RenderParams()
    _abi.lib().s2_default_render_params(p)
    p.spp, p.min_path_length, p.max_path_length, p.flags, p.frame_seed = spp, 2, 3, flags | J, seed
    p.restir_candidates = m
    return p


@pytest.fixture(scope="module")
def lights(device):
    wl = terrain_scene(seed=2, grid=128, spheres=8, sphere_level=2, width=64, height=36, tiles=2,
                       emissive_triangles=256, emissive_sigma=1.0, emissive_power=0.02, emissive_height=(0.4, 0.8),
                       emissive_edge=(0.02, 0.05), sun_radiance=50.0, sun_cone_degrees=5.0, sky_scale=0.02)
    device.upload_scene(wl.scene)
    return wl


def _img(device, wl, p, rad, aov):
    device.render_device(wl.view, p, aov)
    return rad[..., :3].double().cpu().numpy()


def test_power_pick_converges_to_uniform_pick_and_lowers_error(device, lights):
    wl = lights
    rad = torch.zeros((wl.height, wl.width, 4), device="cuda")
    aov = _abi.S2Aovs(rad.data_ptr(), None, None, None, None, None)
    ref = np.stack([_img(device, wl, params(700000 + 4096 * b, 0, spp=4096), rad, aov) for b in range(16)])
    ref_m, ref_v = ref.mean(0), ref.var(0, ddof=1) / 16

    def err(x):
        return float(np.mean((x - ref_m) ** 2 / (ref_m ** 2 + 1e-2)))

    for name, fl in (("NEE", 0), ("RIS", _abi.FLAG_RESTIR_DI)):
        means = np.stack([_img(device, wl, params(100000 + 512 * b, fl | POWER, spp=512), rad, aov) for b in range(16)])
        m, v = means.mean(0), means.var(0, ddof=1) / 16
        z = (m - ref_m) / np.sqrt(v + ref_v + (1e-5 * np.abs(ref_m) + 1e-9) ** 2)
        assert np.mean(np.abs(z) > 5) <= 2e-3, f"{name}: {np.mean(np.abs(z) > 5):.4%} of channels with |z| > 5"
        assert abs(z.mean()) < 0.15, f"{name}: mean z {z.mean():.3f}"
        power = np.stack([_img(device, wl, params(200000 + k, fl | POWER), rad, aov) for k in range(256)])
        uniform = np.stack([_img(device, wl, params(200000 + k, fl), rad, aov) for k in range(256)])
        ratio = err(power) / err(uniform)
        assert ratio < 0.9, f"{name}: power / uniform per-frame error {ratio:.3f}"
