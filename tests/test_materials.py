"""Alpha-masked geometry and normal maps in the oracle (CPU): rays through the masked quad of the
cutout scene pass exactly where the mask's bilinear footprint is 0 and stop where it is 1
(intersection.hlsli:125-146), and ApplyNormalMap (material.hlsli:78-105) changes the packed
shading normals of the bump-mapped walls only."""
import numpy as np
import pytest

from oracle_lib import OracleScene
from stratum2_b200 import _abi
from stratum2_b200.scenegen import cutout_scene

QUAD_Z = 0.2


def quad_rays(mask_shape=(64, 64), n=24):
    """Rays from the camera through points of the masked quad whose 2x2 bilinear texel footprint
    is uniform, with the expected outcome (True: the quad is hit)."""
    wl = cutout_scene(seed=3)
    mask = wl.scene.images[2][:, :, 0]
    h, w = mask.shape
    us = (np.arange(n) + 0.5) / n
    rays, expect, uvs = [], [], []
    for v in us:
        for u in us:
            x, y = u * w - 0.5, v * h - 0.5
            x0, y0 = int(np.floor(x)) % w, int(np.floor(y)) % h
            fp = mask[[y0, y0, (y0 + 1) % h, (y0 + 1) % h], [x0, (x0 + 1) % w, x0, (x0 + 1) % w]]
            if fp.min() != fp.max():
                continue
            p = np.array([-0.7 + 1.4 * u, -0.7 + 1.4 * v, QUAD_Z])
            o = np.array([0.0, 0.0, 3.0])
            d = (p - o) / np.linalg.norm(p - o)
            rays.append([*o, 0.0, *d, np.inf])
            expect.append(fp[0] >= 0.5)
            uvs.append((u, v))
    return wl, np.array(rays, np.float32), np.array(expect)


def test_alpha_mask_decides_hits():
    wl, rays, expect = quad_rays()
    assert expect.sum() > 50 and (~expect).sum() > 20
    osc = OracleScene(wl.scene, 3)
    quad_instance = 6  # 5 walls, the light, then the quad
    for prec in (64, 32):
        h = osc.trace(rays, precision=prec)
        hit_quad = h["instance"] == quad_instance
        np.testing.assert_array_equal(hit_quad, expect)
        behind = h["t"][~expect] > np.linalg.norm(np.array([0, 0, 3.0]) - np.array([0, 0, QUAD_Z])) * 0.99
        assert behind.all()
        any_hit = osc.trace(rays, anyhit=True, precision=prec)
        assert (any_hit["instance"] != 0xFFFFFFFF).all()


def test_alpha_test_off_and_normal_maps_off_change_the_render():
    wl = cutout_scene(seed=3, width=32, height=32)
    osc = OracleScene(wl.scene, 1)
    p = _abi.S2RenderParams()
    _abi.lib().s2_default_render_params(p)
    p.spp, p.min_path_length, p.max_path_length, p.flags = 4, 0, 5, 0
    base = osc.render(wl.view, p, 32, 32)
    p.flags = _abi.FLAG_ALPHA_TEST_OFF
    opaque = osc.render(wl.view, p, 32, 32)
    p.flags = _abi.FLAG_NORMAL_MAPS_OFF
    flat = osc.render(wl.view, p, 32, 32)
    quad = opaque["ids32"][..., 0] == 6
    assert quad.mean() > 0.3
    # holes: pixels that see the quad only when the alpha test is off
    holes = quad & (base["ids32"][..., 0] != 6)
    assert 0.05 < holes.mean() < 0.5
    # normal maps move the packed shading normal on the bump-mapped floor (0) and back wall (2) only
    moved = base["visibility"][..., 1] != flat["visibility"][..., 1]
    ids = base["ids32"][..., 0]
    bumped = (ids == 0) | (ids == 2)
    assert moved[bumped].mean() > 0.9
    assert not moved[~bumped & (ids != 0xFFFFFFFF)].any()
