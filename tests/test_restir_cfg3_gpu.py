"""Screen-space ReSTIR DI at the many-lights workload's parameters: the benchmark terrain carrying
100,000 small emissive triangles of lognormal(0, 2) power, 32 RIS candidates, 1 temporal + 5 spatial
neighbours within 30 pixels, M-cap 20, lights picked in proportion to their power (both estimators),
direct illumination at the primary vertex (path length 2), pixel jitter.  The image is 96x54 instead
of 1920x1080 (same camera and scene; the reference image below needs 65,536 spp per pixel).

The camera plays the workload's closed Catmull-Rom loop (16 views) over and over, reusing across
frames; the frames rendered at the loop's last view average to plain NEE there: a 16 x 4096 spp NEE
image of that view, by a per-pixel z-test and a z-test of the image total over 24 independent
batches of 48 loops (batch means are close to Gaussian; single frames of these lognormal emitters
are heavy tailed).  The per-frame error of the reuse frames is below that of RIS alone."""
import numpy as np
import pytest
import torch

from stratum2_b200 import _abi
from stratum2_b200.scenegen import catmull_rom_views, terrain_scene
from test_restir_screen_gpu import z_check

pytestmark = pytest.mark.gpu
J, PP = _abi.FLAG_PIXEL_JITTER, _abi.FLAG_LIGHT_POWER_PICK
RIS = _abi.FLAG_RESTIR_DI
SCREEN = _abi.FLAG_RESTIR_DI | _abi.FLAG_RESTIR_SCREEN
W, H = 96, 54


def prm(seed, flags, spp=1):
    p = _abi.S2RenderParams()
    _abi.lib().s2_default_render_params(p)
    p.spp, p.min_path_length, p.max_path_length, p.frame_seed = spp, 2, 2, seed
    p.flags = flags | J | PP
    p.restir_candidates, p.restir_spatial, p.restir_spatial_radius, p.restir_max_m = 32, 5, 30.0, 20.0
    return p


def test_cfg3_screen_reuse_unbiased_and_lower_error(device):
    wl = terrain_scene(emissive_triangles=100_000, emissive_sigma=2.0, width=W, height=H)
    device.upload_scene(wl.scene)
    views = catmull_rom_views(W, H, frames=16, seed=11, looping=True)
    last = views[-1]
    rad = torch.zeros((H, W, 4), device="cuda")
    aov = _abi.S2Aovs(rad.data_ptr(), None, None, None, None, None)

    def frame(view, p):
        device.render_device(view, p, aov)
        return rad[..., :3].double().cpu().numpy()

    ref = np.stack([frame(last, prm(700000 + 4096 * b, 0, spp=4096)) for b in range(16)])
    ref_m, ref_v = ref.mean(0), ref.var(0, ddof=1) / len(ref)
    nb, loops = 24, 48
    means, singles, seed = [], [], 50000
    for b in range(nb):
        device.render_device(views[0], prm(1, RIS), aov)  # a call without reuse drops the reservoirs
        acc = []
        for _ in range(loops):
            for v in views:
                device.render_device(v, prm(seed, SCREEN), aov)
                seed += 1
            acc.append(rad[..., :3].double().cpu().numpy())
        means.append(np.mean(acc, axis=0))
        singles += acc[:4]
    means = np.stack(means)
    z_check(means.mean(0), means.var(0, ddof=1) / nb, ref_m, ref_v, "cfg3 screen reuse")
    tot, rtot = means.reshape(nb, -1).sum(1), ref.reshape(len(ref), -1).sum(1)
    zt = (tot.mean() - rtot.mean()) / np.sqrt(tot.var(ddof=1) / nb + rtot.var(ddof=1) / len(rtot))
    assert abs(zt) < 4, f"image total z {zt:.2f} (relative {(tot.mean() - rtot.mean()) / rtot.mean():.4f})"

    def err(x):
        return float(np.mean((x - ref_m) ** 2 / (ref_m ** 2 + 1e-2)))

    ris = np.stack([frame(last, prm(90000 + k, RIS)) for k in range(len(singles))])
    ratio = err(np.stack(singles)) / err(ris)
    print("cfg3 screen reuse / RIS per-frame error", ratio)
    assert ratio < 1.0, f"screen reuse / RIS per-frame error {ratio:.3f}"
