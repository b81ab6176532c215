"""Screen-space ReSTIR DI reuse on the GPU (S2_FLAG_RESTIR_SCREEN; no counterpart in the reference,
which reuses through its world-space hash grid, the S2_FLAG_RESTIR_REUSE mode).

The primary vertex of every path combines its RIS reservoir with the previous call's per-pixel
reservoirs at its reprojected pixel and at random pixels within a radius, by the same two-domain
resampling step as the hash-grid reuse (ReservoirReuse, testrenderer.slang:608-663).  Checks:
  * the first call of a sequence (no previous reservoirs) is the RIS-only render, bit for bit, and
    a sequence is reproducible (no atomics: every pixel's record has one writer);
  * a sequence of reuse frames converges to plain NEE (box: the FP64 golden image; many-lights
    terrain, with a camera moving along a Catmull-Rom path: a 16 x 4096 spp GPU NEE image) by the
    z-test of the other convergence tests;
  * on the many-lights scene it lowers the per-frame error below RIS alone.
"""
from pathlib import Path

import numpy as np
import pytest

from stratum2_b200 import _abi
from stratum2_b200.scenegen import box_scene, catmull_rom_views, terrain_scene

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
J = _abi.FLAG_PIXEL_JITTER
LAM = _abi.FLAG_LAMBERTIAN
RIS = _abi.FLAG_RESTIR_DI
SCREEN = _abi.FLAG_RESTIR_DI | _abi.FLAG_RESTIR_SCREEN


def params(seed, flags, m=4, minl=2, maxl=4, spp=1, spatial=5, radius=30.0, max_m=20.0):
    p = _abi.S2RenderParams()
    _abi.lib().s2_default_render_params(p)
    p.spp, p.min_path_length, p.max_path_length, p.flags, p.frame_seed = spp, minl, maxl, flags, seed
    p.restir_candidates = m
    p.restir_spatial, p.restir_spatial_radius, p.restir_max_m = spatial, radius, max_m
    return p


def lights_wl():
    return terrain_scene(seed=2, grid=128, spheres=8, sphere_level=2, width=64, height=36, tiles=2,
                         emissive_triangles=256, emissive_sigma=1.0, emissive_power=0.02, emissive_height=(0.4, 0.8),
                         emissive_edge=(0.02, 0.05), sun_radiance=50.0, sun_cone_degrees=5.0, sky_scale=0.02)


def img(device, view, wl, p):
    return device.render(view, wl.width, wl.height, params=p).radiance[..., :3].astype(np.float64)


def z_check(m, v, ref, ref_var, tag, mean_z=True):
    z = (m - ref) / np.sqrt(v + ref_var + (1e-5 * np.abs(ref) + 1e-9) ** 2)
    frac = np.mean(np.abs(z) > 5)
    assert frac <= 2e-3, f"{tag}: {frac:.4%} of pixel channels with |z| > 5"
    if mean_z:
        assert abs(z.mean()) < 0.15, f"{tag}: mean z {z.mean():.3f}"


def total_check(seq_means, ref, ref_var, tag, bound=4.0):
    """Bias test on the image total: the sequences' totals are independent (one per sequence),
    where the pixels of one sequence are not (spatial reuse shares reservoirs between neighbours,
    so an image-wide mean of per-pixel z scores measured -0.15 to +0.29 between seed sets of an
    unbiased estimator)."""
    totals = seq_means[..., :3].sum(axis=(1, 2, 3))
    ref_total, ref_total_var = ref[..., :3].sum(), ref_var[..., :3].sum()
    t = (totals.mean() - ref_total) / np.sqrt(totals.var(ddof=1) / len(totals) + ref_total_var)
    assert abs(t) < bound, f"{tag}: image total {totals.mean():.6g} against {ref_total:.6g} (t = {t:.2f})"


@pytest.fixture(scope="module")
def lights(device):
    wl = lights_wl()
    device.upload_scene(wl.scene)
    return wl


def test_first_call_is_ris_and_sequences_reproduce(device, lights):
    wl = lights
    device.upload_scene(wl.scene)
    img(device, wl.view, wl, params(1, RIS | J | LAM))  # a call without the flag drops the reservoirs
    a = img(device, wl.view, wl, params(2, SCREEN | J | LAM))
    b = img(device, wl.view, wl, params(2, RIS | J | LAM))
    np.testing.assert_array_equal(a, b)
    seqs = []
    for rep in range(2):
        img(device, wl.view, wl, params(1, RIS | J | LAM))
        seqs.append([img(device, wl.view, wl, params(10 + k, SCREEN | J | LAM)) for k in range(4)])
    for x, y in zip(*seqs):
        np.testing.assert_array_equal(x, y)
    assert not np.array_equal(seqs[0][3], img(device, wl.view, wl, params(13, RIS | J | LAM)))


def test_box_screen_reuse_converges_to_fp64_golden(device):
    wl = box_scene(seed=1, width=64, height=64)
    device.upload_scene(wl.scene)
    gold = np.load(GOLDEN / "box_64x64_fp64_16384spp.npz")
    means = []
    for b in range(16):
        img(device, wl.view, wl, params(1, RIS | J | LAM, minl=2, maxl=5))
        means.append(np.mean([img(device, wl.view, wl, params(30000 + 256 * b + k, SCREEN | J | LAM, minl=2, maxl=5))
                              for k in range(256)], axis=0))
    means = np.stack(means)
    z_check(means.mean(0), means.var(0, ddof=1) / 16, gold["mean"], gold["var_of_mean"], "box screen reuse", mean_z=False)
    total_check(means, gold["mean"], gold["var_of_mean"], "box screen reuse")


def test_many_lights_moving_camera_unbiased_and_lower_error(device, lights):
    """The camera plays a closed 16-frame Catmull-Rom loop over and over, reusing across frames; the
    frames rendered at the loop's last view, 128 per batch, average to plain NEE there (32 batches:
    per-pixel z-test and a z-test of the image total), and their per-frame error is below RIS alone
    at that view (0.60 of it measured on B200; reuse acts at the primary vertex only, the indirect
    bounces of these paths up to length 4 keep their noise).  Frames of one batch are correlated through the reservoirs they share, so
    batches need many frames before their means are close enough to Gaussian for the z-test (with
    64, the skew of single-frame estimates already shows as a mean z of -0.1 for RIS alone)."""
    import torch
    wl = lights
    device.upload_scene(wl.scene)
    views = catmull_rom_views(wl.width, wl.height, frames=16, seed=5, looping=True)
    last = views[-1]
    ref = np.stack([img(device, last, wl, params(500000 + 4096 * b, J | LAM, spp=4096)) for b in range(16)])
    ref_m, ref_v = ref.mean(0), ref.var(0, ddof=1) / 16
    rad = torch.zeros((wl.height, wl.width, 4), device="cuda")
    aov = _abi.S2Aovs(rad.data_ptr(), None, None, None, None, None)
    means, singles = [], []
    seed = 40000
    nb = 32
    for b in range(nb):
        device.render_device(views[0], params(1, RIS | J | LAM), aov)  # start without reservoirs
        acc = []
        for loop in range(128):
            for v in views:
                device.render_device(v, params(seed, SCREEN | J | LAM), aov)
                seed += 1
            acc.append(rad[..., :3].double().cpu().numpy())
        means.append(np.mean(acc, axis=0))
        singles += acc[:8]
    means = np.stack(means)
    z_check(means.mean(0), means.var(0, ddof=1) / nb, ref_m, ref_v, "moving-camera screen reuse")
    tot, rtot = means.reshape(nb, -1).sum(1), ref.reshape(len(ref), -1).sum(1)
    zt = (tot.mean() - rtot.mean()) / np.sqrt(tot.var(ddof=1) / nb + rtot.var(ddof=1) / len(rtot))
    assert abs(zt) < 4, f"image total z {zt:.2f} (relative {(tot.mean() - rtot.mean()) / rtot.mean():.4f})"

    def err(x):
        return float(np.mean((x - ref_m) ** 2 / (ref_m ** 2 + 1e-2)))

    ris = np.stack([img(device, last, wl, params(90000 + k, RIS | J | LAM)) for k in range(len(singles))])
    ratio = err(np.stack(singles)) / err(ris)
    assert ratio < 0.75, f"screen reuse / RIS per-frame error {ratio:.3f}"


def test_screen_reuse_argument_errors(device, lights):
    wl = lights
    device.upload_scene(wl.scene)
    p = params(1, SCREEN | J | _abi.FLAG_RADIANCE_CACHE)
    with pytest.raises(_abi.S2Error) as e:
        device.render_views([wl.view], p)
    assert e.value.code == _abi.S2_ERR_UNSUPPORTED
    p = params(1, SCREEN | J)
    p.flags |= _abi.FLAG_RESTIR_REUSE
    with pytest.raises(_abi.S2Error) as e:
        device.render(wl.view, wl.width, wl.height, params=p)
    assert e.value.code == _abi.S2_ERR_INVALID
    p = params(1, SCREEN | J, spatial=33)
    with pytest.raises(_abi.S2Error) as e:
        device.render(wl.view, wl.width, wl.height, params=p)
    assert e.value.code == _abi.S2_ERR_INVALID


def test_screen_reuse_with_visibility_first_call_and_reproducible(device, lights):
    """S2_FLAG_RESTIR_REUSE_VISIBILITY on the screen-space reuse: the first call equals the plain
    screen-space first call (no previous reservoirs), and sequences reproduce bit for bit."""
    wl = lights
    device.upload_scene(wl.scene)
    V = _abi.FLAG_RESTIR_REUSE_VISIBILITY
    img(device, wl.view, wl, params(1, RIS | J))  # drop previous reservoirs
    a = img(device, wl.view, wl, params(40, SCREEN | LAM | J))
    img(device, wl.view, wl, params(1, RIS | J))
    b = img(device, wl.view, wl, params(40, SCREEN | V | LAM | J))
    np.testing.assert_allclose(b, a, rtol=1e-6, atol=1e-9)
    seqs = []
    for _ in range(2):
        img(device, wl.view, wl, params(1, RIS | J))
        seqs.append(np.stack([img(device, wl.view, wl, params(50 + k, SCREEN | V | LAM | J)) for k in range(4)]))
    np.testing.assert_array_equal(seqs[0], seqs[1])


def views_img(device, views, p):
    res, _ = device.render_views(views, p)
    return np.stack([r.radiance[..., :3].astype(np.float64) for r in res])


def test_batched_screen_reuse_first_call_and_reproducible(device, lights):
    """s2_render_views with screen-space reuse: one reservoir per pixel of every view.  Without
    previous reservoirs the call is the RIS-only batched render bit for bit, and sequences
    reproduce bit for bit."""
    wl = lights
    device.upload_scene(wl.scene)
    views = [wl.view, wl.view]
    a = views_img(device, views, params(60, RIS | LAM | J))
    b = views_img(device, views, params(60, SCREEN | LAM | J))  # the RIS-only call dropped the reservoirs
    np.testing.assert_array_equal(a, b)
    seqs = []
    for _ in range(2):
        views_img(device, views, params(1, RIS | J))
        seqs.append(np.stack([views_img(device, views, params(70 + k, SCREEN | LAM | J)) for k in range(4)]))
    np.testing.assert_array_equal(seqs[0], seqs[1])


def test_batched_screen_reuse_matches_single_view_sequence(device):
    """Batched screen-space reuse over two views of the box runs the single-view estimator in each
    view: over 8 sequences of 64 calls, each view's mean image equals the s2_render sequence's with
    the same seeds (accumulation order differs: fixed-point totals against float), and the two
    views equal each other.  The single-view estimator itself is checked against the FP64 golden
    image by test_box_screen_reuse_converges_to_fp64_golden.  (With spatial reuse, neighbouring
    pixels share reservoirs, so an image-wide mean z is far from normal with few sequences: it
    measured -0.12 and +0.29 for two seed sets of the single-view test, in the batched path
    alike.)"""
    wl = box_scene(seed=1, width=64, height=64)
    device.upload_scene(wl.scene)
    views = [wl.view, wl.view]
    single, both = [], []
    for b in range(8):
        img(device, wl.view, wl, params(1, RIS | J | LAM, minl=2, maxl=5))
        single.append(np.mean([img(device, wl.view, wl, params(30000 + 256 * b + k, SCREEN | J | LAM, minl=2, maxl=5))
                               for k in range(64)], axis=0))
        views_img(device, views, params(1, RIS | J | LAM, minl=2, maxl=5))
        both.append(np.mean([views_img(device, views, params(30000 + 256 * b + k, SCREEN | J | LAM, minl=2, maxl=5))
                             for k in range(64)], axis=0))
    single, both = np.stack(single), np.stack(both)  # [b, H, W, 3], [b, view, H, W, 3]
    np.testing.assert_allclose(both[:, 0], both[:, 1], rtol=1e-6, atol=1e-9)
    m, ms = both[:, 0].mean(0), single.mean(0)
    assert abs(m.sum() / ms.sum() - 1) < 1e-3, (m.sum(), ms.sum())
    assert np.mean(np.abs(m - ms)) < 1e-3 * np.mean(ms), np.mean(np.abs(m - ms)) / np.mean(ms)


def test_batched_screen_reuse_of_different_views_matches_each_single_view(device):
    """Two views that differ in camera and extent (64x64 and 48x32) in one batched call: each view
    keeps its own reservoirs (its slice of the per-pixel records), so over 4 sequences of 32 calls
    each view's mean image equals its own s2_render sequence's with the same seeds, within the
    accumulation-order tolerance of the identical-view test."""
    from stratum2_b200.scene import make_view
    wl = box_scene(seed=1, width=64, height=64)
    device.upload_scene(wl.scene)
    rot = np.array([[0.9659258, 0.0, 0.258819], [0.0, 1.0, 0.0], [-0.258819, 0.0, 0.9659258]])
    other = make_view((0.6, 0.1, 2.6), 48, 32, 45.0, rot)
    views = [wl.view, other]
    extents = [(64, 64), (48, 32)]

    def single(view, wh, seed0):
        w, h = wh
        device.render(view, w, h, params=params(1, RIS | J | LAM, minl=2, maxl=5))
        return np.mean([device.render(view, w, h, params=params(seed0 + k, SCREEN | J | LAM, minl=2, maxl=5))
                        .radiance[..., :3].astype(np.float64) for k in range(32)], axis=0)

    singles = [[], []]
    batched = [[], []]
    for b in range(4):
        seed0 = 50000 + 128 * b
        for v in range(2):
            singles[v].append(single(views[v], extents[v], seed0))
        device.render_views(views, params(1, RIS | J | LAM, minl=2, maxl=5))
        calls = [device.render_views(views, params(seed0 + k, SCREEN | J | LAM, minl=2, maxl=5))[0] for k in range(32)]
        for v in range(2):
            batched[v].append(np.mean([c[v].radiance[..., :3].astype(np.float64) for c in calls], axis=0))
    for v in range(2):
        m, ms = np.mean(batched[v], axis=0), np.mean(singles[v], axis=0)
        assert m.shape == (extents[v][1], extents[v][0], 3)
        assert abs(m.sum() / ms.sum() - 1) < 1e-3, (v, m.sum(), ms.sum())
        assert np.mean(np.abs(m - ms)) < 1e-3 * np.mean(ms), (v, np.mean(np.abs(m - ms)) / np.mean(ms))
