"""ReSTIR DI reuse through the world-space hash grid on the GPU (S2_FLAG_RESTIR_REUSE,
testrenderer.slang:608-726, hashgrid.hlsli:14-119).

The grid build lists each cell's records in an order fixed by their content (a scan of the cell
counters and a sort by cell and record hash, where the reference keeps the atomic append order), so
reuse sequences are reproducible bit for bit; the estimator is checked statistically:
  * the first call of a sequence (no previous grid) is the RIS-only render, bit for bit, and
    repeating a sequence repeats its images;
  * a sequence of reuse frames converges to plain NEE (box: the FP64 golden image; many-lights
    terrain: a 16 x 4096 spp GPU NEE image) by the same z-test as the other convergence tests;
  * on the many-lights scene (256 emitters, power lognormal(0, 1), Lambertian, direct light only)
    with 4 candidates, reuse lowers the per-frame error, and the ratio of per-frame errors
    (reuse / RIS-only, about 0.8) agrees with the oracle's restatement of the same estimator.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle_lib import OracleScene
from stratum2_b200 import _abi
from stratum2_b200.scenegen import box_scene, terrain_scene

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
J = _abi.FLAG_PIXEL_JITTER
RIS = _abi.FLAG_RESTIR_DI
REUSE = _abi.FLAG_RESTIR_DI | _abi.FLAG_RESTIR_REUSE


def params(seed, flags, m=32, minl=1, maxl=6, spp=1):
    p = _abi.S2RenderParams()
    _abi.lib().s2_default_render_params(p)
    p.spp, p.min_path_length, p.max_path_length, p.flags, p.frame_seed = spp, minl, maxl, flags, seed
    p.restir_candidates = m
    return p


LAM = _abi.FLAG_LAMBERTIAN


def lights_wl():
    return terrain_scene(seed=2, grid=128, spheres=8, sphere_level=2, width=64, height=36, tiles=2,
                         emissive_triangles=256, emissive_sigma=1.0, emissive_power=0.02, emissive_height=(0.4, 0.8),
                         emissive_edge=(0.02, 0.05), sun_radiance=50.0, sun_cone_degrees=5.0, sky_scale=0.02)


@pytest.fixture(scope="module")
def lights(device):
    wl = lights_wl()
    device.upload_scene(wl.scene)
    return wl


def render(device, wl, p):
    return device.render(wl.view, wl.width, wl.height, params=p)


def frames(device, wl, flags, m, seed0, n, minl=1, maxl=6):
    out = []
    for k in range(n):
        out.append(render(device, wl, params(seed0 + k, flags | J, m, minl, maxl)).radiance[..., :3].astype(np.float64))
    return np.stack(out)


def z_check(m, v, ref, ref_var, tag):
    z = (m - ref) / np.sqrt(v + ref_var + (1e-5 * np.abs(ref) + 1e-9) ** 2)
    frac = np.mean(np.abs(z) > 5)
    assert frac <= 2e-3, f"{tag}: {frac:.4%} of pixel channels with |z| > 5"
    assert abs(z.mean()) < 0.15, f"{tag}: mean z {z.mean():.3f}"


def test_reuse_sequences_are_reproducible(device, lights):
    wl = lights
    seqs = []
    for _ in range(2):
        device.upload_scene(wl.scene)  # a fresh render state: no previous grid
        seqs.append(frames(device, wl, REUSE, 4, 300, 5))
    np.testing.assert_array_equal(seqs[0], seqs[1])


def test_first_reuse_call_is_ris_and_reuse_changes_later_calls(device, lights):
    wl = lights
    device.upload_scene(wl.scene)  # a fresh render state has no previous grid
    a = render(device, wl, params(1, REUSE | J, 4))
    b = render(device, wl, params(1, RIS | J, 4))
    np.testing.assert_array_equal(a.radiance, b.radiance)
    assert a.stats.kernel_launches == b.stats.kernel_launches + 3  # grid build: scan, keys, sort
    render(device, wl, params(2, REUSE | J, 4))
    c = render(device, wl, params(3, REUSE | J, 4))
    d = render(device, wl, params(3, RIS | J, 4))
    assert not np.array_equal(c.radiance, d.radiance)
    assert c.stats.nan_count == 0 and np.isfinite(c.radiance).all()


def test_box_reuse_converges_to_fp64_golden(device):
    wl = box_scene(seed=1, width=64, height=64)
    device.upload_scene(wl.scene)
    gold = np.load(GOLDEN / "box_64x64_fp64_16384spp.npz")
    means = [frames(device, wl, REUSE | _abi.FLAG_LAMBERTIAN, 4, 10000 + 256 * b, 256, 2, 5).mean(0)
             for b in range(16)]
    means = np.stack(means)
    z_check(means.mean(0), means.var(0, ddof=1) / 16, gold["mean"], gold["var_of_mean"], "box reuse")


def test_many_lights_reuse_unbiased(device, lights):
    wl = lights
    device.upload_scene(wl.scene)
    ref = np.stack([render(device, wl, params(500000 + 4096 * b, J | LAM, minl=2, maxl=4, spp=4096))
                    .radiance[..., :3].astype(np.float64) for b in range(16)])
    render(device, wl, params(1, RIS | J, 2))  # drop any previous grid
    means = np.stack([frames(device, wl, REUSE | LAM, 2, 20000 + 256 * b, 256, 2, 4).mean(0) for b in range(16)])
    z_check(means.mean(0), means.var(0, ddof=1) / 16, ref.mean(0), ref.var(0, ddof=1) / 16, "many-lights reuse")


def test_many_lights_reuse_lowers_error_like_the_oracle(device, lights):
    wl = lights
    device.upload_scene(wl.scene)
    ref = render(device, wl, params(700000, J | LAM, minl=2, maxl=2, spp=65536)).radiance[..., :3].astype(np.float64)

    def err(imgs):
        return float(np.mean((imgs - ref) ** 2 / (ref ** 2 + 1e-2)))

    ris = frames(device, wl, RIS | LAM, 4, 90000, 2048, 2, 2)
    render(device, wl, params(89999, REUSE | LAM | J, 4, 2, 2))
    reu = frames(device, wl, REUSE | LAM, 4, 90000, 2048, 2, 2)
    gpu_ratio = err(reu) / err(ris)
    osc = OracleScene(wl.scene, 1)
    o = {}
    for name, fl in (("ris", RIS), ("reuse", REUSE)):
        osc.render(wl.view, params(89999, fl | LAM | J, 4, 2, 2), wl.width, wl.height)
        o[name] = np.stack([osc.render(wl.view, params(90000 + k, fl | LAM | J, 4, 2, 2), wl.width, wl.height)["mean"]
                            for k in range(768)])
    oracle_ratio = err(o["reuse"]) / err(o["ris"])
    assert gpu_ratio < 0.92, f"reuse / RIS per-frame error {gpu_ratio:.3f}"
    assert abs(gpu_ratio - oracle_ratio) < 0.15 * oracle_ratio, (gpu_ratio, oracle_ratio)


def test_reuse_argument_errors(device, lights):
    wl = lights
    device.upload_scene(wl.scene)
    p = params(1, REUSE | J, 4)
    p.restir_grid_cell_size = float("nan")
    with pytest.raises(_abi.S2Error) as e:
        render(device, wl, p)
    assert e.value.code == _abi.S2_ERR_INVALID
    with pytest.raises(_abi.S2Error) as e:
        device.render_views([wl.view], p)
    assert e.value.code == _abi.S2_ERR_INVALID


def batched(device, views, flags, m, seed, minl=1, maxl=6):
    res, _ = device.render_views(views, params(seed, flags | J, m, minl, maxl))
    return np.stack([r.radiance[..., :3].astype(np.float64) for r in res])


def test_batched_reuse_first_call_is_ris(device, lights):
    """s2_render_views with hash-grid reuse: without a previous grid the call is the RIS-only
    batched render, bit for bit (fixed-point pixel totals)."""
    wl = lights
    device.upload_scene(wl.scene)
    views = [wl.view, wl.view]
    a = batched(device, views, RIS | LAM, 4, 77, 2, 4)
    b = batched(device, views, REUSE | LAM, 4, 77, 2, 4)  # the RIS-only call dropped the grids
    np.testing.assert_array_equal(a, b)


def test_batched_reuse_sequence_unbiased(device, lights):
    """Several views reuse one world-space grid per call, as TestRenderer's views do: a sequence
    of batched reuse calls over two views converges to plain NEE in both views."""
    wl = lights
    device.upload_scene(wl.scene)
    ref = np.stack([render(device, wl, params(600000 + 4096 * b, J | LAM, minl=2, maxl=4, spp=4096))
                    .radiance[..., :3].astype(np.float64) for b in range(16)])
    views = [wl.view, wl.view]
    means = []
    for b in range(16):
        batched(device, views, RIS | LAM, 4, 40000 + 1000 * b - 1, 2, 4)  # new sequence
        means.append(np.stack([batched(device, views, REUSE | LAM, 4, 40000 + 1000 * b + k, 2, 4)
                               for k in range(128)]).mean(0))
    means = np.stack(means)  # [batch, view, H, W, 3]
    for v in range(2):
        z_check(means[:, v].mean(0), means[:, v].var(0, ddof=1) / 16, ref.mean(0), ref.var(0, ddof=1) / 16,
                f"batched reuse, view {v}")


VIS = _abi.FLAG_RESTIR_REUSE_VISIBILITY


def test_reuse_visibility_first_call_equals_plain_reuse(device, lights):
    """gReSTIR_DI_Reuse_Visibility without a previous grid: zeroing W of an occluded canonical
    sample and adding the traced result directly change nothing, so the first call equals plain
    reuse's first call (the RIS-only render)."""
    wl = lights
    device.upload_scene(wl.scene)
    render(device, wl, params(1, RIS | J, 4))  # drop any previous grid
    a = render(device, wl, params(31, REUSE | LAM | J, 4, 2, 4)).radiance
    render(device, wl, params(1, RIS | J, 4))
    b = render(device, wl, params(31, REUSE | VIS | LAM | J, 4, 2, 4)).radiance
    np.testing.assert_allclose(b, a, rtol=1e-6, atol=1e-9)


def test_reuse_visibility_matches_the_oracle(device, lights):
    """The reuse-visibility estimator (testrenderer.slang:611-616, 689-694, 742-743) is biased near
    shadow boundaries (reused samples are weighted with unshadowed target pdfs), so the check is
    against the oracle's restatement of the same estimator, not against plain NEE: 16 sequences
    of 64 frames each, batch means compared by the z-test, and the per-frame error ratio to RIS
    alone within 15 % of the oracle's."""
    wl = lights
    device.upload_scene(wl.scene)
    osc = OracleScene(wl.scene, 1)
    ref = render(device, wl, params(700000, J | LAM, minl=2, maxl=2, spp=65536)).radiance[..., :3].astype(np.float64)

    def err(imgs):
        return float(np.mean((imgs - ref) ** 2 / (ref ** 2 + 1e-2)))

    g, o = [], []
    for b in range(16):
        s0 = 300000 + 1000 * b
        render(device, wl, params(s0 - 1, RIS | J, 4))  # drop the grid: a new sequence
        g.append(frames(device, wl, REUSE | VIS | LAM, 4, s0, 64, 2, 2))
        osc.render(wl.view, params(s0 - 1, RIS | LAM | J, 4, 2, 2), wl.width, wl.height)
        o.append(np.stack([osc.render(wl.view, params(s0 + k, REUSE | VIS | LAM | J, 4, 2, 2), wl.width, wl.height)["mean"]
                           for k in range(64)]))
    g, o = np.stack(g), np.stack(o)
    gm, om = g.mean(1), o.mean(1)
    z = (gm.mean(0) - om.mean(0)) / np.sqrt(gm.var(0, ddof=1) / 16 + om.var(0, ddof=1) / 16 + 1e-12)
    assert np.mean(np.abs(z) > 5) <= 2e-3, f"{np.mean(np.abs(z) > 5):.4%} of pixel channels with |z| > 5"
    assert abs(z.mean()) < 0.15, z.mean()
    ris = frames(device, wl, RIS | LAM, 4, 90000, 1024, 2, 2)
    gpu_ratio = err(g.reshape(-1, *g.shape[2:])) / err(ris)
    ris_o = np.stack([osc.render(wl.view, params(90000 + k, RIS | LAM | J, 4, 2, 2), wl.width, wl.height)["mean"]
                      for k in range(1024)])
    oracle_ratio = err(o.reshape(-1, *o.shape[2:])) / err(ris_o)
    assert gpu_ratio < 0.92, gpu_ratio
    assert abs(gpu_ratio - oracle_ratio) < 0.15 * oracle_ratio, (gpu_ratio, oracle_ratio)
