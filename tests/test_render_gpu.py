"""Parity of the wavefront path tracer (CUDA) with the FP64 oracle.

Same-seed tests: the GPU and the oracle draw the same random numbers per (pixel, sample) (the
reference's counter-based pcg4d stream, or PCG32), so they trace the same paths up to
floating-point divergence of individual paths.  The floor of that divergence is set by the
reference's own path-state packing: ray directions are stored octahedral SNORM16
(testrenderer.slang:119-122), so a 1e-7 rounding difference flips ~2% of direction components by
one 3e-5 rad step, which occasionally moves a hit across a small triangle's edge; and at pixel
centres the symmetric box puts diagonal pixels' camera rays exactly on its corner seams, where
float and double tie-break differently.  The oracle's own FP32 build diverges from its FP64 build
at the same rate (~0.06% of samples with pixel jitter, ~0.15% at pixel centres).  The tests render
one sample per call for 16 seeds on both sides and require that at most 1% of (pixel, sample)
values differ by more than 1e-3 relative (+1e-4 absolute) in any channel.

Convergence tests: the mean of 16 independent GPU batches against a committed FP64 oracle image
rendered with disjoint seeds (tests/golden/make_golden.py).  Per pixel channel
z = (gpu - oracle) / sqrt(var_gpu + var_oracle) with var_gpu from the 16 batches (t, 15 dof):
|z| > 5 for at most 0.1% of channels, |mean z| < 0.1 (no global bias), and relMSE below 1e-3
(box) or twice the noise floor the two estimators' variances predict (terrain: sun and glossy spheres
give a high relative per-sample variance).  The parity terrain uses a sun of radiance 50 over a
5 degree cone: the benchmark's 5e3 sun over 0.5 degrees makes per-pixel estimates heavy-tailed
(rare sun reflections), which no z-test at these sample counts can assess.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle_lib import OracleScene
from stratum2_b200 import _abi
from stratum2_b200.metrics import relmse
from stratum2_b200.scenegen import box_scene, terrain_scene

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def make_params(spp, min_len, max_len, flags, seed=0, restir_m=32):
    p = _abi.S2RenderParams()
    _abi.lib().s2_default_render_params(p)
    p.spp, p.min_path_length, p.max_path_length, p.flags, p.frame_seed = spp, min_len, max_len, flags, seed
    p.restir_candidates = restir_m
    return p


def box_wl():
    return box_scene(seed=1, width=64, height=64)


def terrain_wl():
    return terrain_scene(seed=2, grid=128, spheres=8, sphere_level=2, width=64, height=36, tiles=2, area_lights=2,
                         sun_radiance=50.0, sun_cone_degrees=5.0)


def per_sample_divergence(device, osc, wl, p, n=16):
    """Fraction of (pixel, sample) radiance values where GPU and oracle differ by more than
    1e-3 relative + 1e-4 absolute in any channel, over n single-sample renders."""
    seed0 = p.frame_seed
    bad = 0
    for k in range(n):
        p.spp, p.frame_seed = 1, seed0 + k
        g = device.render(wl.view, wl.width, wl.height, params=p).radiance[..., :3].astype(np.float64)
        o = osc.render(wl.view, p, wl.width, wl.height)["mean"]
        bad += int((np.abs(g - o) > 1e-3 * np.abs(o) + 1e-4).any(-1).sum())
    p.frame_seed = seed0
    return bad / (n * wl.width * wl.height)


def assert_same_seed(device, osc, wl, p, tag=""):
    d = per_sample_divergence(device, osc, wl, p)
    assert d <= 0.01, f"{tag}: {d:.4%} of samples diverge"


def batches(device, wl, p, n, spp, seed0):
    """Mean and variance of the mean over n independent GPU renders of `spp` samples."""
    imgs = []
    for b in range(n):
        p.spp, p.frame_seed = spp, seed0 + b * spp
        imgs.append(device.render(wl.view, wl.width, wl.height, params=p).radiance[..., :3].astype(np.float64))
    imgs = np.stack(imgs)
    return imgs.mean(0), imgs.var(0, ddof=1) / n


def assert_converged(mean_a, var_a, mean_b, var_b, relmse_max, tag=""):
    # variance floored at float resolution (directly visible sky has zero variance in both)
    z = (mean_a - mean_b) / np.sqrt(var_a + var_b + (1e-5 * np.abs(mean_b) + 1e-9) ** 2)
    frac = np.mean(np.abs(z) > 5)
    assert frac <= 1e-3, f"{tag}: {frac:.4%} of pixel channels with |z| > 5"
    assert abs(z.mean()) < 0.1, f"{tag}: mean z {z.mean():.3f} (bias)"
    rm = relmse(mean_a, mean_b)
    assert rm <= relmse_max, f"{tag}: relMSE {rm} > {relmse_max}"


@pytest.fixture(scope="module")
def box(device):
    wl = box_wl()
    device.upload_scene(wl.scene)
    return wl, OracleScene(wl.scene, 1)


J = _abi.FLAG_PIXEL_JITTER


@pytest.mark.parametrize("min_len,max_len,extra", [(2, 5, 0), (2, 5, J), (0, 3, J), (1, 8, _abi.FLAG_PCG32 | J),
                                                   (2, 5, _abi.FLAG_NO_NEE | J), (2, 5, _abi.FLAG_NO_RR | J)])
def test_box_same_seed_matches_fp64_oracle(device, box, min_len, max_len, extra):
    wl, osc = box
    device.upload_scene(wl.scene)
    p = make_params(1, min_len, max_len, _abi.FLAG_LAMBERTIAN | extra, seed=7)
    assert_same_seed(device, osc, wl, p, f"min{min_len} max{max_len} flags{extra}")
    p.spp = 16
    g = device.render(wl.view, wl.width, wl.height, params=p)
    assert g.stats.extension_rays > 0 and g.stats.nan_count == 0


def test_box_aovs_match_oracle(device, box):
    wl, osc = box
    device.upload_scene(wl.scene)
    p = make_params(2, 2, 5, _abi.FLAG_LAMBERTIAN, seed=0)
    g = device.render(wl.view, wl.width, wl.height, params=p)
    o = osc.render(wl.view, p, wl.width, wl.height)
    ids_same = (g.ids32 == o["ids32"]).all(-1)
    assert ids_same.mean() > 0.999
    np.testing.assert_array_equal(g.visibility[..., 0][ids_same], o["visibility"][..., 0][ids_same])
    np.testing.assert_allclose(g.albedo[ids_same], o["albedo"][ids_same], atol=1e-6)
    np.testing.assert_allclose(g.depth[..., 0][ids_same], o["depth"][..., 0][ids_same], rtol=1e-3)
    np.testing.assert_allclose(g.prev_uv[ids_same], o["prev_uv"][ids_same], atol=1e-4)
    # packed shading normals agree to within one SNORM16 step per component
    a = g.visibility[..., 1][ids_same].astype(np.int64)
    b = o["visibility"][..., 1][ids_same].astype(np.int64)
    dx = np.abs(((a & 0xFFFF) ^ 0x8000) - ((b & 0xFFFF) ^ 0x8000))
    dy = np.abs(((a >> 16) ^ 0x8000) - ((b >> 16) ^ 0x8000))
    assert dx.max() <= 1 and dy.max() <= 1


def test_exposure_deterministic_and_accumulate(device, box):
    wl, _ = box
    device.upload_scene(wl.scene)
    p = make_params(8, 2, 5, _abi.FLAG_LAMBERTIAN, seed=3)
    a = device.render(wl.view, wl.width, wl.height, params=p)
    b = device.render(wl.view, wl.width, wl.height, params=p)
    np.testing.assert_array_equal(a.radiance, b.radiance)  # deterministic (no atomics on the accumulators)
    p.exposure = 1.5
    c = device.render(wl.view, wl.width, wl.height, params=p)
    np.testing.assert_allclose(c.radiance[..., :3], a.radiance[..., :3] * 2 ** 1.5, rtol=1e-6)
    # two progressive calls of 8 spp == one call of 16 spp
    p16 = make_params(16, 2, 5, _abi.FLAG_LAMBERTIAN, seed=3)
    p16.wave_paths = 8 * wl.width * wl.height
    full = device.render(wl.view, wl.width, wl.height, params=p16)
    p8 = make_params(8, 2, 5, _abi.FLAG_LAMBERTIAN, seed=3)
    device.render(wl.view, wl.width, wl.height, params=p8)
    p8b = make_params(8, 2, 5, _abi.FLAG_LAMBERTIAN | _abi.FLAG_ACCUMULATE, seed=11)
    acc = device.render(wl.view, wl.width, wl.height, params=p8b)
    np.testing.assert_allclose(acc.radiance, full.radiance, rtol=1e-6, atol=1e-7)


def test_box_converges_to_fp64_golden(device, box):
    wl, _ = box
    device.upload_scene(wl.scene)
    gold = np.load(GOLDEN / "box_64x64_fp64_16384spp.npz")
    p = make_params(1, 2, 5, _abi.FLAG_LAMBERTIAN | J)
    m, v = batches(device, wl, p, 16, 256, seed0=0)  # 4096 spp in total
    assert_converged(m, v, gold["mean"], gold["var_of_mean"], 1e-3, "box 4096 spp")


@pytest.fixture(scope="module")
def terrain(device):
    wl = terrain_wl()
    return wl, OracleScene(wl.scene, 1)


@pytest.mark.parametrize("extra", [0, _abi.FLAG_REFERENCE_ENV_MIS, _abi.FLAG_SHADING_NORMALS_OFF,
                                   _abi.FLAG_ENV_FOOTPRINT_PDF])
def test_terrain_disney_env_same_seed(device, terrain, extra):
    wl, osc = terrain
    device.upload_scene(wl.scene)
    p = make_params(1, 1, 6, extra | J, seed=5)
    assert_same_seed(device, osc, wl, p, f"terrain flags{extra}")


@pytest.mark.parametrize("extra", [0, _abi.FLAG_ENV_FOOTPRINT_PDF])
def test_terrain_converges_to_fp64_golden(device, terrain, extra):
    """With the reference's texel pdf and with the footprint pdf (an unbiased change of the
    environment's sampling density: the same expected image)."""
    wl, _ = terrain
    device.upload_scene(wl.scene)
    gold = np.load(GOLDEN / "terrain_64x36_fp64_131072spp.npz")
    p = make_params(1, 1, 6, J | extra)
    m, v = batches(device, wl, p, 16, 4096, seed0=0)  # 65536 spp in total
    floor = np.mean((v + gold["var_of_mean"]) / (gold["mean"] ** 2 + 1e-2))
    assert_converged(m, v, gold["mean"], gold["var_of_mean"], max(1e-3, 2 * floor), "terrain 65536 spp")


@pytest.mark.parametrize("scene_name", ["box", "terrain"])
def test_restir_di_same_seed_and_unbiased(device, box, terrain, scene_name):
    wl, osc = box if scene_name == "box" else terrain
    base = _abi.FLAG_LAMBERTIAN if scene_name == "box" else 0
    minl, maxl = (2, 5) if scene_name == "box" else (1, 6)
    device.upload_scene(wl.scene)
    p = make_params(1, minl, maxl, base | _abi.FLAG_RESTIR_DI | J, seed=9, restir_m=8)
    assert_same_seed(device, osc, wl, p, f"restir {scene_name}")
    # RIS with M candidates converges to the same image as plain NEE
    mr, vr = batches(device, wl, make_params(1, minl, maxl, base | _abi.FLAG_RESTIR_DI | J, restir_m=8), 16, 512, 100)
    mn, vn = batches(device, wl, make_params(1, minl, maxl, base | J), 16, 512, 20000)
    floor = np.mean((vr + vn) / (mn ** 2 + 1e-2))
    assert_converged(mr, vr, mn, vn, 3 * floor, f"restir vs nee {scene_name}")


def test_invalid_arguments_return_errors(device, box):
    wl, _ = box
    device.upload_scene(wl.scene)
    p = make_params(0, 2, 5, _abi.FLAG_LAMBERTIAN)
    with pytest.raises(_abi.S2Error) as e:
        device.render(wl.view, wl.width, wl.height, params=p)
    assert e.value.code == _abi.S2_ERR_INVALID
    p = make_params(1, 2, 300, _abi.FLAG_LAMBERTIAN)
    with pytest.raises(_abi.S2Error):
        device.render(wl.view, wl.width, wl.height, params=p)
