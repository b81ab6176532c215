"""Post-processing on the GPU against the numpy oracle (oracle/post_oracle.py, the reference's
temporal_accumulation.slang and tonemap.slang restated in float64):
  * s2_tonemap: every TonemapMode, with and without gamma (standard sRGB and the reference's
    rgbToSrgb), albedo modulation and exposure, within float32 rounding;
  * s2_temporal_accumulate: four frames rendered by s2_render with a moving camera, accumulated
    with reprojection (instance, normal and depth checks), albedo demodulation, shadow hysteresis,
    a history limit, and without reprojection, within float32 rounding."""
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

from stratum2_b200 import _abi
from stratum2_b200.scene import make_view, transform_trs
from stratum2_b200.scenegen import box_scene

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import post_oracle as po  # noqa: E402

pytestmark = pytest.mark.gpu


def _close(a, b, rtol, atol):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    both_nan = np.isnan(a) & np.isnan(b)
    np.testing.assert_allclose(np.where(both_nan, 0, a), np.where(both_nan, 0, b), rtol=rtol, atol=atol)


@pytest.mark.parametrize("mode", range(11))
def test_tonemap_matches_oracle(device, mode):
    rng = np.random.default_rng(mode)
    H, W = 48, 64
    img = np.concatenate([rng.lognormal(-1, 1.5, (H, W, 3)), np.ones((H, W, 1))], -1).astype(np.float32)
    img[0, :4, :3] = 0.0
    alb = rng.uniform(0, 1, (H, W, 4)).astype(np.float32)
    x, a = torch.from_numpy(img).cuda(), torch.from_numpy(alb).cuda()
    out = torch.zeros_like(x)
    for flags in (0, _abi.TONEMAP_GAMMA, _abi.TONEMAP_GAMMA_REFERENCE):
        for use_alb in (False, True):
            for exposure in (0.0, 1.5):
                p = _abi.S2TonemapParams(mode, exposure, flags, 0)
                device.tonemap(W, H, p, x.data_ptr(), out.data_ptr(), a.data_ptr() if use_alb else None)
                ref = po.tonemap(img, mode, exposure, gamma=bool(flags & 1), gamma_reference=bool(flags & 2),
                                 albedo=alb if use_alb else None)
                _close(out.cpu().numpy(), ref, rtol=2e-4, atol=2e-5)


def _frames(device, n=4, W=48, H=40):
    wl = box_scene(seed=1, n_random=60, width=W, height=H)
    device.upload_scene(wl.scene)
    bufs = []
    prev = None
    for k in range(n):
        pos = (0.03 * k, 0.01 * k, 3.0)
        view = make_view(pos, W, H, 40.0, prev_camera_to_world=prev)
        prev = transform_trs(pos, np.eye(3))
        t = {"radiance": torch.zeros((H, W, 4), device="cuda"), "albedo": torch.zeros((H, W, 4), device="cuda"),
             "vis": torch.zeros((H, W, 2), dtype=torch.int32, device="cuda"), "depth": torch.zeros((H, W, 4), device="cuda"),
             "prev_uv": torch.zeros((H, W, 2), device="cuda")}
        aov = _abi.S2Aovs(t["radiance"].data_ptr(), t["albedo"].data_ptr(), t["vis"].data_ptr(), t["depth"].data_ptr(),
                          t["prev_uv"].data_ptr(), None)
        p = device.default_params()
        p.spp, p.min_path_length, p.max_path_length, p.flags, p.frame_seed = 2, 0, 4, _abi.FLAG_PIXEL_JITTER, 100 + 2 * k
        device.render_device(view, p, aov)
        bufs.append((view, t, aov))
    return bufs


@pytest.mark.parametrize("flags,limit", [
    (_abi.TEMPORAL_REPROJECT | _abi.TEMPORAL_CHECK_NORMAL | _abi.TEMPORAL_CHECK_DEPTH, 0),
    (_abi.TEMPORAL_REPROJECT | _abi.TEMPORAL_DEMODULATE_ALBEDO | _abi.TEMPORAL_SHADOW_HYSTERESIS, 3),
    (0, 0),
])
def test_temporal_accumulation_matches_oracle(device, flags, limit):
    frames = _frames(device)
    H, W = frames[0][1]["radiance"].shape[:2]
    color = torch.zeros((H, W, 4), device="cuda")
    moments = torch.zeros((H, W, 2), device="cuda")
    prev = None
    for k, (view, t, aov) in enumerate(frames):
        tp = device.default_temporal_params()
        tp.flags = flags | (_abi.TEMPORAL_RESET if k == 0 else 0)
        tp.history_limit = limit
        device.temporal_accumulate(view, tp, aov, color.data_ptr(), moments.data_ptr())
        host = {name: v.cpu().numpy() for name, v in t.items()}
        vis = host["vis"].view(np.uint32)
        oc, om = po.temporal_accumulate(host["radiance"], host["albedo"], vis, host["depth"], host["prev_uv"], prev, flags,
                                        history_limit=limit)
        _close(color.cpu().numpy(), oc, rtol=2e-4, atol=1e-6)
        _close(moments.cpu().numpy(), om, rtol=2e-4, atol=1e-6)
        prev = {"color": color.cpu().numpy().astype(np.float64), "moments": moments.cpu().numpy().astype(np.float64),
                "vis": vis, "depth": host["depth"]}
    if flags & _abi.TEMPORAL_REPROJECT:
        # reprojection found history for most pixels of the moving view
        assert np.mean(color.cpu().numpy()[..., 3] > 1.5) > 0.5


def test_post_argument_errors(device):
    frames = _frames(device, n=1)
    view, t, aov = frames[0]
    tp = device.default_temporal_params()
    bad = _abi.S2Aovs(t["radiance"].data_ptr(), None, None, None, None, None)
    with pytest.raises(_abi.S2Error):
        device.temporal_accumulate(view, tp, bad, t["radiance"].data_ptr())
    with pytest.raises(_abi.S2Error):
        device.tonemap(8, 8, _abi.S2TonemapParams(99, 0.0, 0, 0), t["radiance"].data_ptr(), t["albedo"].data_ptr())


@pytest.mark.parametrize("kernel,iterations,tap", [(_abi.SVGF_KERNEL_BOX3, 3, 0), (_abi.SVGF_KERNEL_ATROUS, 2, 1),
                                                   (_abi.SVGF_KERNEL_BOX5_SUBSAMPLED, 3, 2)])
def test_svgf_matches_oracle(device, kernel, iterations, tap):
    """s2_svgf_filter after two accumulated frames against the oracle's estimate_variance and
    atrous passes (and the history tap's colour copy)."""
    frames = _frames(device, n=2, W=24, H=20)
    H, W = 20, 24
    color = torch.zeros((H, W, 4), device="cuda")
    moments = torch.zeros((H, W, 2), device="cuda")
    tp = device.default_temporal_params()
    for k, (view, t, aov) in enumerate(frames):
        tp.flags = (tp.flags | _abi.TEMPORAL_RESET) if k == 0 else (tp.flags & ~_abi.TEMPORAL_RESET)
        device.temporal_accumulate(view, tp, aov, color.data_ptr(), moments.data_ptr())
    view, t, aov = frames[-1]
    sp = device.default_svgf_params()
    sp.kernel, sp.iterations, sp.history_tap, sp.history_limit = kernel, iterations, tap, 2
    out = torch.zeros((H, W, 4), device="cuda")
    device.svgf_filter(view, sp, aov, out.data_ptr())
    host = {name: v.cpu().numpy() for name, v in t.items()}
    vis = host["vis"].view(np.uint32)
    c, m = color.cpu().numpy().astype(np.float64), moments.cpu().numpy().astype(np.float64)
    img = [po.svgf_variance(c, m, vis, host["depth"], sp.flags, history_limit=2, boost=sp.variance_boost_length), None]
    tapped = None
    for i in range(iterations):
        img[(i + 1) % 2] = po.svgf_atrous(img[i % 2], vis, host["depth"], i, kernel, sp.flags, sp.sigma_luminance_boost)
        if i + 1 == tap:
            tapped = img[0].copy()  # copy_rgb reads filter image 0 whichever image the pass wrote
    _close(out.cpu().numpy(), img[iterations % 2], rtol=2e-3, atol=1e-5)
    if tap:
        # the history's colour now holds filter image 0's rgb (the next accumulation reads it)
        h2 = torch.zeros((H, W, 4), device="cuda")
        tp.flags = 0  # no reprojection: the next frame blends with the history in place
        device.temporal_accumulate(view, tp, aov, h2.data_ptr())
        prev_rgb = tapped[..., :3]
        cur = host["radiance"][..., :3].astype(np.float64)
        n = c[..., 3:4] + 1
        _close(h2.cpu().numpy()[..., :3], prev_rgb + (cur - prev_rgb) / n, rtol=2e-3, atol=1e-5)
