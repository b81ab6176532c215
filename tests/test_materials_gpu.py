"""Alpha-masked geometry (gAlphaTest, intersection.hlsli:125-146) and normal maps (gNormalMaps,
material.hlsli:78-105) on the GPU, against the oracle, on the cutout scene (normal-mapped textured
floor and back wall, an alpha-masked quad in front of random triangles).

The alpha test compares a bilinear texture tap with the cutoff, so a hit within float rounding of
the cutoff may be decided differently by the GPU and the FP32 oracle; the trace tests allow 0.1%
of rays to differ, and rays through uniform texel footprints must agree exactly.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle_lib import OracleScene, camera_rays, random_rays
from stratum2_b200 import _abi
from stratum2_b200.scenegen import cutout_scene
from test_materials import quad_rays
from test_render_gpu import assert_converged, assert_same_seed, batches, make_params

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
J = _abi.FLAG_PIXEL_JITTER


@pytest.fixture(scope="module")
def cutout(device):
    wl = cutout_scene(seed=3, width=64, height=64)
    device.upload_scene(wl.scene)
    return wl, OracleScene(wl.scene, 3)


def test_alpha_mask_decides_hits(device, cutout):
    wl, osc = cutout
    device.upload_scene(wl.scene)
    _, rays, expect = quad_rays()
    h = device.trace(rays)
    np.testing.assert_array_equal(h["instance"] == 6, expect)
    a = device.trace(rays, anyhit=True)
    assert (a["instance"] != 0xFFFFFFFF).all()


@pytest.mark.parametrize("anyhit", [False, True])
def test_trace_matches_fp32_oracle(device, cutout, anyhit):
    wl, osc = cutout
    device.upload_scene(wl.scene)
    rays = np.concatenate([camera_rays(wl.view, 256, 256), random_rays(100000, seed=5, lo=-0.95, hi=0.95)])
    g = device.trace(rays, anyhit=anyhit)
    o = osc.trace(rays, anyhit=anyhit, precision=32)
    if anyhit:
        same = (g["instance"] == 0xFFFFFFFF) == (o["instance"] == 0xFFFFFFFF)
    else:
        same = (g["instance"] == o["instance"]) & (g["primitive"] == o["primitive"])
    assert (~same).mean() <= 1e-3, f"{(~same).mean():.4%} of rays differ"
    if not anyhit:
        np.testing.assert_array_equal(g["t"][same].view(np.uint32), o["t"][same].astype(np.float32).view(np.uint32))


@pytest.mark.parametrize("extra", [J, _abi.FLAG_ALPHA_TEST_OFF | J, _abi.FLAG_NORMAL_MAPS_OFF | J,
                                   _abi.FLAG_LAMBERTIAN | J, 0])
def test_cutout_same_seed_matches_fp64_oracle(device, cutout, extra):
    wl, osc = cutout
    device.upload_scene(wl.scene)
    p = make_params(1, 0, 5, extra, seed=13)
    assert_same_seed(device, osc, wl, p, f"cutout flags {extra}")


def test_normal_mapped_visibility_aov(device, cutout):
    wl, osc = cutout
    device.upload_scene(wl.scene)
    p = make_params(1, 0, 5, 0, seed=2)
    g = device.render(wl.view, wl.width, wl.height, params=p)
    o = osc.render(wl.view, p, wl.width, wl.height)
    ids_same = (g.ids32 == o["ids32"]).all(-1)
    assert ids_same.mean() > 0.995
    bumped = ids_same & np.isin(g.ids32[..., 0], (0, 2))
    assert bumped.mean() > 0.2
    a = g.visibility[..., 1][ids_same].astype(np.int64)
    b = o["visibility"][..., 1][ids_same].astype(np.int64)
    dx = np.abs(((a & 0xFFFF) ^ 0x8000) - ((b & 0xFFFF) ^ 0x8000))
    dy = np.abs(((a >> 16) ^ 0x8000) - ((b >> 16) ^ 0x8000))
    assert np.mean((dx > 1) | (dy > 1)) <= 1e-3
    flat = device.render(wl.view, wl.width, wl.height, params=make_params(1, 0, 5, _abi.FLAG_NORMAL_MAPS_OFF, seed=2))
    moved = g.visibility[..., 1] != flat.visibility[..., 1]
    assert moved[bumped].mean() > 0.9


def test_cutout_converges_to_fp64_golden(device, cutout):
    wl, _ = cutout
    device.upload_scene(wl.scene)
    gold = np.load(GOLDEN / "cutout_64x64_fp64_16384spp.npz")
    m, v = batches(device, wl, make_params(1, 0, 5, J), 16, 256, seed0=0)
    floor = np.mean((v + gold["var_of_mean"]) / (gold["mean"] ** 2 + 1e-2))
    assert_converged(m, v, gold["mean"], gold["var_of_mean"], max(1e-3, 2 * floor), "cutout 4096 spp")


def test_cutout_restir_reuse_converges(device, cutout):
    wl, _ = cutout
    device.upload_scene(wl.scene)
    gold = np.load(GOLDEN / "cutout_64x64_fp64_16384spp.npz")
    flags = _abi.FLAG_RESTIR_DI | _abi.FLAG_RESTIR_REUSE | J
    means = []
    for b in range(16):
        acc = 0.0
        for f in range(128):
            p = make_params(1, 0, 5, flags, seed=30000 + 128 * b + f, restir_m=4)
            acc = acc + device.render(wl.view, wl.width, wl.height, params=p).radiance[..., :3].astype(np.float64)
        means.append(acc / 128)
    means = np.stack(means)
    m, v = means.mean(0), means.var(0, ddof=1) / 16
    z = (m - gold["mean"]) / np.sqrt(v + gold["var_of_mean"] + (1e-5 * np.abs(gold["mean"]) + 1e-9) ** 2)
    assert np.mean(np.abs(z) > 5) <= 2e-3 and abs(z.mean()) < 0.15, (np.mean(np.abs(z) > 5), z.mean())
