"""Traversal parity on the benchmark's own BVH: the terrain workload at full size (1024^2 terrain
grid, 2,093,058 triangles, plus 64 instanced level-5 icospheres, 3,403,778 triangles, 507,592 BVH8
nodes), the scene every bench frame traces.  About one million seeded rays: every 4th camera ray of
the 1920x1080 benchmark view (518,400), 400,000 random rays inside the scene's box and 81,600 with
tmin > 0 and a finite tmax.  Criteria as in test_trace_gpu.py: bit-identical hits against the
oracle's FP32 replica of the watertight test; against FP64, ids equal except equal-t ties (< 1e-4
of the rays) and t within 1e-5 relative except a few grazing hits on instanced icospheres (< 2e-5 of
the hits, all within 1e-4); any-hit visibility equal to the replica's; and the
counted walk's node and triangle fetches equal the CPU BVH8 walker's (the byte model behind the
traversal roofline)."""
import ctypes as C

import numpy as np
import pytest

from oracle_lib import OracleScene, camera_rays, oracle, random_rays
from stratum2_b200.scenegen import terrain_scene

pytestmark = pytest.mark.gpu
INV = 0xFFFFFFFF


@pytest.fixture(scope="module")
def cfg2(device):
    wl = terrain_scene()
    device.upload_scene(wl.scene)
    assert device.bvh_stats.triangle_count == 3_403_778
    osc = OracleScene(wl.scene, 3)
    cam = camera_rays(wl.view, wl.width, wl.height)[::4]
    rnd = random_rays(400_000, seed=21, lo=-1.0, hi=1.0)
    seg = random_rays(81_600, seed=22, lo=-1.0, hi=1.0)
    seg[:, 3] = 0.01
    seg[:, 7] = 0.5
    rays = np.ascontiguousarray(np.concatenate([cam, rnd, seg]), np.float32)
    assert len(rays) == 1_000_000
    return wl, osc, rays


def test_cfg2_closest_hit_bit_exact_vs_fp32_oracle(device, cfg2):
    wl, osc, rays = cfg2
    g = device.trace(rays)
    o = osc.trace(rays, precision=32)
    hit = g["instance"] != INV
    assert hit.mean() > 0.3
    np.testing.assert_array_equal(g["instance"], o["instance"])
    np.testing.assert_array_equal(g["primitive"], o["primitive"])
    np.testing.assert_array_equal(g["t"][hit], o["t"][hit].astype(np.float32))
    np.testing.assert_array_equal(g["b1"][hit], o["b1"][hit].astype(np.float32))
    np.testing.assert_array_equal(g["b2"][hit], o["b2"][hit].astype(np.float32))


def test_cfg2_closest_hit_vs_fp64_oracle(device, cfg2):
    wl, osc, rays = cfg2
    g = device.trace(rays)
    o = osc.trace(rays, precision=64)
    same = (g["instance"] == o["instance"]) & (g["primitive"] == o["primitive"])
    both = (g["instance"] != INV) & (o["instance"] != INV)
    mismatch = ~same
    assert mismatch.mean() < 1e-4, f"{mismatch.sum()} id mismatches of {len(rays)}"
    assert np.all(both[mismatch]), "a ray hit in one implementation and missed in the other"
    rel = np.abs(g["t"][both].astype(np.float64) - o["t"][both]) / np.maximum(o["t"][both], 5e-2)
    # The float32 world-space vertices of instanced meshes carry ~1 ulp of rounding, which grazing
    # hits on the small icosphere triangles amplify (measured: 3 of 447,073 hits above 1e-5, all on
    # icospheres at t < 0.05, at most 4.5e-5; the FP32 replica reproduces them bit for bit).
    assert (rel > 1e-5).mean() < 2e-5, (rel > 1e-5).sum()
    assert rel.max() < 1e-4, rel.max()


def test_cfg2_anyhit_matches_fp32_oracle(device, cfg2):
    wl, osc, rays = cfg2
    g = device.trace(rays, anyhit=True)
    o = osc.trace(rays, anyhit=True, precision=32)
    np.testing.assert_array_equal(g["instance"] != INV, o["instance"] != INV)


def test_cfg2_fetch_counts_match_cpu_bvh8_walker(device, cfg2):
    wl, osc, rays = cfg2
    sub = np.ascontiguousarray(rays[::20], np.float32)
    nodes, tris = device.get_bvh()
    L = oracle()
    L.oracle_bvh8_trace.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p, C.c_void_p]
    h, cnt = device.trace(sub, counted=True)
    oh = np.zeros((len(sub), 5), np.uint32)
    oc = np.zeros((len(sub), 2), np.uint32)
    L.oracle_bvh8_trace(nodes.ctypes.data, tris.ctypes.data, sub.ctypes.data, len(sub), 0, oh.ctypes.data, oc.ctypes.data)
    np.testing.assert_array_equal(cnt, oc)
    np.testing.assert_array_equal(h["instance"], oh[:, 1])
    np.testing.assert_array_equal(h["t"].view(np.uint32), oh[:, 0])
