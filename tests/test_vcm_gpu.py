"""Vertex connection and merging (s2_render_vcm: the reference's VCM renderer, VCM.cpp:370-620 and
vcm.slang:880-1238, SmallVCM's techniques with the dVCM / dVC / dVM MIS quantities).

* The unbiased algorithms (path tracing, light tracing, BPT with and without the light vertex cache)
  converge to the FP64 path-traced golden image of the box scene (paths of 2..5 segments, box pixel
  filter), by the z-test of the other convergence tests: their MIS weights sum to one.
* Each BPT technique alone, unweighted (the reference's debug-path mode), converges to the image of
  the paths of its length that path tracing renders: every technique's pdf and throughput
  bookkeeping is checked without MIS.
* Merging is consistent: BPM, VCM and PPM approach the golden image as the merge radius shrinks.
* Direct illumination by resampled reservoirs (the reference's gDIReservoirFlags eRIS and eReuse,
  vcm.slang:251-390) and the resampled light-vertex-cache connection (gLVCReservoirFlags eRIS and
  eReuse, vcm.slang:568-736) leave these images unchanged in expectation: path tracing and BPT with
  them, with and without the reuse of the previous iteration's reservoirs through the hash grids,
  converge to the same golden image.
"""
from pathlib import Path

import numpy as np
import pytest

from stratum2_b200 import _abi
from stratum2_b200.api import Device
from stratum2_b200.scenegen import box_scene

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
W = H = 64


def vparams(algo, iters, seed, vcm_flags=0, fraction=1.0, radius=0.025, first=0, lengths=(2, 5), di_m=None,
            lvc_max_m=None):
    p = Device.default_vcm_params()
    if di_m is not None:
        p.di_candidates = di_m
    if lvc_max_m is not None:
        p.lvc_max_m = lvc_max_m
    p.algorithm, p.iterations, p.frame_seed = algo, iters, seed
    p.min_path_length, p.max_path_length = lengths
    p.flags = _abi.FLAG_LAMBERTIAN
    p.vcm_flags = vcm_flags
    p.light_path_fraction = fraction
    p.merge_radius_factor = radius
    p.first_iteration = first
    return p


def batches(device, view, n, iters, seed0, **kw):
    return np.stack([device.render_vcm(view, W, H, vparams(iters=iters, seed=seed0 + iters * b, **kw)).radiance[..., :3]
                     .astype(np.float64) for b in range(n)])


def zstats(img, ref, ref_v):
    m, v = img.mean(0), img.var(0, ddof=1) / img.shape[0]
    z = (m - ref) / np.sqrt(v + ref_v + (1e-5 * np.abs(ref) + 1e-9) ** 2)
    return z, (m.sum() - ref.sum()) / ref.sum()


@pytest.fixture(scope="module")
def box(device):
    wl = box_scene(seed=1, width=W, height=H)
    device.upload_scene(wl.scene)
    gold = np.load(GOLDEN / "box_64x64_fp64_16384spp.npz")
    return wl, gold["mean"], gold["var_of_mean"]


@pytest.mark.parametrize("algo,vcm_flags,fraction", [
    (_abi.VCM_PATH_TRACE, 0, 1.0),
    (_abi.VCM_LIGHT_TRACE, 0, 2.0),
    (_abi.VCM_BPT, 0, 1.0),
    (_abi.VCM_BPT, _abi.VCM_FLAG_LIGHT_VERTEX_CACHE, 1.0),
])
def test_unbiased_algorithms_converge_to_golden(device, box, algo, vcm_flags, fraction):
    wl, ref, ref_v = box
    device.upload_scene(wl.scene)
    img = batches(device, wl.view, 16, 512, 1000 + 100000 * algo + 7 * vcm_flags, algo=algo, vcm_flags=vcm_flags,
                  fraction=fraction)
    z, rel = zstats(img, ref, ref_v)
    assert np.mean(np.abs(z) > 5) <= 2e-3, f"{np.mean(np.abs(z) > 5):.4%} of pixel channels with |z| > 5"
    assert abs(z.mean()) < 0.15, z.mean()
    assert abs(rel) < 5e-3, rel


@pytest.mark.parametrize("cam,light", [(4, 0), (3, 1), (2, 2), (1, 3)])
def test_each_bpt_technique_unweighted_matches_path_tracing(device, box, cam, light):
    """Paths of exactly 3 segments: emission hit (4, 0), direct illumination (3, 1), connection of
    the first camera and first light vertices (2, 2) and light tracing (1, 3), each alone with MIS
    weight 1, against s2_render's path tracer restricted to length 3."""
    wl, _, _ = box
    device.upload_scene(wl.scene)
    pt = Device.default_params()
    pt.min_path_length = pt.max_path_length = 3
    pt.flags = _abi.FLAG_LAMBERTIAN | _abi.FLAG_PIXEL_JITTER
    pt.spp = 2048
    ref = []
    for b in range(16):
        pt.frame_seed = 700000 + 2048 * b
        ref.append(device.render(wl.view, W, H, params=pt).radiance[..., :3].astype(np.float64))
    ref = np.stack(ref)
    img = []
    for b in range(16):
        p = vparams(_abi.VCM_BPT, 1024, 5000 + 1024 * b, lengths=(3, 3),
                    vcm_flags=_abi.VCM_FLAG_DEBUG_PATHS | _abi.VCM_FLAG_DEBUG_UNWEIGHTED)
        p.debug_camera_vertices, p.debug_light_vertices = cam, light
        img.append(device.render_vcm(wl.view, W, H, p).radiance[..., :3].astype(np.float64))
    img = np.stack(img)
    # Unweighted, the connection technique has unbounded variance where the two vertices meet (its
    # 1/d^2 term), so per-pixel means over 16 batches are heavy-tailed: the z-test runs on 8x8
    # pixel blocks, and the image total must agree within 1 %.
    blk = lambda a: a.reshape(a.shape[0], H // 8, 8, W // 8, 8, 3).sum((2, 4))
    bi, br = blk(img), blk(ref)
    z, rel = zstats(bi, br.mean(0), br.var(0, ddof=1) / 16)
    assert np.mean(np.abs(z) > 5) <= 1e-2, f"{np.mean(np.abs(z) > 5):.4%} of block channels with |z| > 5"
    assert abs(z.mean()) < 0.5, z.mean()
    assert abs(rel) < 1e-2, rel


@pytest.mark.parametrize("algo", [_abi.VCM_BPM, _abi.VCM_VCM, _abi.VCM_PPM])
def test_merging_converges_as_the_radius_shrinks(device, box, algo):
    """Density estimation loses energy where the merge disc overhangs an edge, so the merging-only
    algorithms are biased by an amount that shrinks with the radius (measured on this scene: BPM
    -2.7 % of the image total at 0.04 of the scene radius, -1.1 % at 0.01).  VCM weights merging
    against the connection techniques, and at 0.01 passes the unbiased z-test."""
    wl, ref, ref_v = box
    device.upload_scene(wl.scene)
    errs = []
    for radius in (0.04, 0.01):
        img = batches(device, wl.view, 8, 256, 9000 + 1000 * algo, algo=algo, radius=radius)
        errs.append(abs((img.mean(0) - ref).sum() / ref.sum()))
    assert errs[1] < errs[0] and errs[1] < 1.6e-2, errs
    if algo == _abi.VCM_VCM:
        z, rel = zstats(img, ref, ref_v)
        assert np.mean(np.abs(z) > 5) <= 2e-3, f"{np.mean(np.abs(z) > 5):.4%} of pixel channels with |z| > 5"
        assert abs(z.mean()) < 0.15, z.mean()
        assert abs(rel) < 5e-3, rel


def test_vcm_reproducible_aovs_and_argument_checks(device, box):
    wl, _, _ = box
    device.upload_scene(wl.scene)
    for algo, fl in ((_abi.VCM_VCM, 0), (_abi.VCM_BPT, _abi.VCM_FLAG_LIGHT_VERTEX_CACHE)):
        a = device.render_vcm(wl.view, W, H, vparams(algo, 4, 11, vcm_flags=fl))
        b = device.render_vcm(wl.view, W, H, vparams(algo, 4, 11, vcm_flags=fl))
        np.testing.assert_array_equal(a.radiance, b.radiance)
        assert a.stats.extension_rays > 0 and a.stats.shadow_rays > 0 and a.stats.nan_count == 0
        assert a.stats.paths == 4 * W * H
    # first-hit AOVs: the closed box is hit everywhere, ids match the path tracer's first hits
    r = device.render_vcm(wl.view, W, H, vparams(_abi.VCM_BPT, 1, 3))
    assert np.all(np.isfinite(r.depth[..., 0])) and np.all(r.depth[..., 0] > 0)
    assert np.all(r.ids32[..., 0] != 0xffffffff)
    with pytest.raises(_abi.S2Error) as e:
        device.render_vcm(wl.view, W, H, vparams(6, 1, 0))
    assert e.value.code == _abi.S2_ERR_INVALID
    with pytest.raises(_abi.S2Error) as e:
        device.render_vcm(wl.view, W, H, vparams(_abi.VCM_VCM, 1, 0, vcm_flags=_abi.VCM_FLAG_LIGHT_VERTEX_CACHE))
    assert e.value.code == _abi.S2_ERR_UNSUPPORTED
    p = vparams(_abi.VCM_BPT, 1, 0)
    p.flags |= _abi.FLAG_RESTIR_DI
    with pytest.raises(_abi.S2Error) as e:
        device.render_vcm(wl.view, W, H, p)
    assert e.value.code == _abi.S2_ERR_UNSUPPORTED
    p = vparams(_abi.VCM_BPT, 1, 0, fraction=0.0)
    with pytest.raises(_abi.S2Error) as e:
        device.render_vcm(wl.view, W, H, p)
    assert e.value.code == _abi.S2_ERR_INVALID


@pytest.mark.parametrize("algo,vcm_flags", [
    (_abi.VCM_BPT, _abi.VCM_FLAG_LIGHT_VERTEX_CACHE | _abi.VCM_FLAG_LVC_RIS),
    (_abi.VCM_BPT, _abi.VCM_FLAG_LIGHT_VERTEX_CACHE | _abi.VCM_FLAG_LVC_RIS | _abi.VCM_FLAG_DI_RIS),
    (_abi.VCM_PATH_TRACE, _abi.VCM_FLAG_DI_RIS),
    (_abi.VCM_BPT, _abi.VCM_FLAG_DI_RIS),
    (_abi.VCM_PATH_TRACE, _abi.VCM_FLAG_DI_RIS | _abi.VCM_FLAG_DI_REUSE),
    (_abi.VCM_BPT, _abi.VCM_FLAG_LIGHT_VERTEX_CACHE | _abi.VCM_FLAG_DI_RIS | _abi.VCM_FLAG_DI_REUSE),
    (_abi.VCM_BPT, _abi.VCM_FLAG_LIGHT_VERTEX_CACHE | _abi.VCM_FLAG_LVC_RIS | _abi.VCM_FLAG_LVC_REUSE),
    (_abi.VCM_BPT, _abi.VCM_FLAG_LIGHT_VERTEX_CACHE | _abi.VCM_FLAG_LVC_RIS | _abi.VCM_FLAG_LVC_REUSE |
     _abi.VCM_FLAG_DI_RIS | _abi.VCM_FLAG_DI_REUSE),
])
def test_di_reservoirs_converge_to_golden(device, box, algo, vcm_flags):
    """Resampled direct illumination (8 candidates per camera vertex) and resampled light-vertex-cache
    connections, with and without reuse, are unbiased: the image converges to the FP64 golden.  With
    reuse, neighbouring pixels share reservoirs, so the bias check is on the image total (one value
    per independent batch) and the per-pixel z-test only bounds the outliers."""
    wl, ref, ref_v = box
    device.upload_scene(wl.scene)
    device.render_vcm(wl.view, W, H, vparams(algo, 1, 1))  # a call without reuse drops old reservoirs
    img = batches(device, wl.view, 16, 256, 5000 + 100000 * algo + 7 * vcm_flags, algo=algo, vcm_flags=vcm_flags, di_m=8)
    z, rel = zstats(img, ref, ref_v)
    assert np.mean(np.abs(z) > 5) <= 2e-3, f"{np.mean(np.abs(z) > 5):.4%} of pixel channels with |z| > 5"
    totals = img.sum(axis=(1, 2, 3))
    t = (totals.mean() - ref.sum()) / np.sqrt(totals.var(ddof=1) / len(totals) + ref_v.sum())
    assert abs(t) < 4.0, (t, rel)
    if not vcm_flags & (_abi.VCM_FLAG_DI_REUSE | _abi.VCM_FLAG_LVC_REUSE):
        assert abs(z.mean()) < 0.15, z.mean()


def test_di_reservoirs_reproducible_and_argument_checks(device, box):
    """Reservoir sequences reproduce bit for bit (the grid is built by a sort on cell and record
    content), reuse changes the image, and the flags are checked."""
    wl, _, _ = box
    device.upload_scene(wl.scene)
    fl = _abi.VCM_FLAG_DI_RIS | _abi.VCM_FLAG_DI_REUSE
    seqs = []
    for _ in range(2):
        device.render_vcm(wl.view, W, H, vparams(_abi.VCM_BPT, 1, 1))  # drops the grids
        seqs.append(np.stack([device.render_vcm(wl.view, W, H, vparams(_abi.VCM_BPT, 2, 40 + 2 * k, vcm_flags=fl)).radiance
                              for k in range(3)]))
    np.testing.assert_array_equal(seqs[0], seqs[1])
    ris = device.render_vcm(wl.view, W, H, vparams(_abi.VCM_BPT, 2, 44, vcm_flags=_abi.VCM_FLAG_DI_RIS)).radiance
    assert not np.array_equal(seqs[0][2], ris)  # the third call reused the second's reservoirs
    lvc = _abi.VCM_FLAG_LIGHT_VERTEX_CACHE | _abi.VCM_FLAG_LVC_RIS
    for bad in (vparams(_abi.VCM_BPT, 1, 0, vcm_flags=_abi.VCM_FLAG_DI_REUSE),
                vparams(_abi.VCM_BPT, 1, 0, vcm_flags=_abi.VCM_FLAG_DI_RIS, di_m=0),
                vparams(_abi.VCM_BPT, 1, 0, vcm_flags=_abi.VCM_FLAG_LVC_RIS),
                vparams(_abi.VCM_BPT, 1, 0, vcm_flags=_abi.VCM_FLAG_LIGHT_VERTEX_CACHE | _abi.VCM_FLAG_LVC_REUSE),
                vparams(_abi.VCM_BPT, 1, 0, vcm_flags=lvc | _abi.VCM_FLAG_LVC_REUSE, lvc_max_m=0.0)):
        with pytest.raises(_abi.S2Error) as e:
            device.render_vcm(wl.view, W, H, bad)
        assert e.value.code == _abi.S2_ERR_INVALID


def test_lvc_reservoir_reuse_reproducible(device, box):
    """LVC reservoir sequences reproduce bit for bit, a call reuses the previous call's reservoirs
    (its image differs from resampling alone), and a call without reuse drops them."""
    wl, _, _ = box
    device.upload_scene(wl.scene)
    lvc = _abi.VCM_FLAG_LIGHT_VERTEX_CACHE | _abi.VCM_FLAG_LVC_RIS
    fl = lvc | _abi.VCM_FLAG_LVC_REUSE
    seqs = []
    for _ in range(2):
        device.render_vcm(wl.view, W, H, vparams(_abi.VCM_BPT, 1, 1))  # drops the grids
        seqs.append(np.stack([device.render_vcm(wl.view, W, H, vparams(_abi.VCM_BPT, 2, 60 + 2 * k, vcm_flags=fl)).radiance
                              for k in range(3)]))
    np.testing.assert_array_equal(seqs[0], seqs[1])
    assert np.all(np.isfinite(seqs[0]))
    ris = device.render_vcm(wl.view, W, H, vparams(_abi.VCM_BPT, 2, 64, vcm_flags=lvc)).radiance
    assert not np.array_equal(seqs[0][2], ris)  # the third call reused the second's reservoirs
    # after a call without reuse the first reuse call has no history: its first iteration resamples
    # alone, so it differs from the same call made with the history of a reuse call
    device.render_vcm(wl.view, W, H, vparams(_abi.VCM_BPT, 1, 1))
    fresh = device.render_vcm(wl.view, W, H, vparams(_abi.VCM_BPT, 2, 60, vcm_flags=fl)).radiance
    np.testing.assert_array_equal(fresh, seqs[0][0])


def test_reservoir_grids_grown_for_a_larger_view_carry_no_history(device, box):
    """A call that needs larger reservoir grids than the previous one (here a 64x64 view after a
    32x32 one) reallocates them, so the reservoirs of the smaller call are gone: its first
    iteration must resample without history, exactly as after a call without reuse."""
    from stratum2_b200.scene import make_view
    wl, _, _ = box
    device.upload_scene(wl.scene)
    small = make_view((0.0, 0.0, 3.0), 32, 32, 40.0)
    fl = (_abi.VCM_FLAG_LIGHT_VERTEX_CACHE | _abi.VCM_FLAG_LVC_RIS | _abi.VCM_FLAG_LVC_REUSE |
          _abi.VCM_FLAG_DI_RIS | _abi.VCM_FLAG_DI_REUSE)
    device.render_vcm(small, 32, 32, vparams(_abi.VCM_BPT, 2, 70, vcm_flags=fl, di_m=8))  # grids sized for 32x32
    grown = device.render_vcm(wl.view, W, H, vparams(_abi.VCM_BPT, 2, 80, vcm_flags=fl, di_m=8)).radiance
    device.render_vcm(wl.view, W, H, vparams(_abi.VCM_BPT, 1, 1))  # drops the grids
    fresh = device.render_vcm(wl.view, W, H, vparams(_abi.VCM_BPT, 2, 80, vcm_flags=fl, di_m=8)).radiance
    assert np.all(np.isfinite(grown))
    np.testing.assert_array_equal(grown, fresh)
