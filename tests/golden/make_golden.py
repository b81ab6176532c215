"""Generates the FP64 oracle reference images used by the GPU convergence tests.

    python tests/golden/make_golden.py

Each fixture is an .npz with the per-pixel mean radiance and the variance of that mean, rendered
by the FP64 oracle (oracle/oracle.cpp) at high sample counts with frame seeds disjoint from the
ones the GPU tests use, with jittered pixel positions (the converged image is then the box-filtered
pixel integral, which has no exact ray/edge ties).  Scenes come from stratum2_b200.scenegen with fixed seeds.
"""
from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE.parent))

from oracle_lib import OracleScene  # noqa: E402
from stratum2_b200 import _abi  # noqa: E402
from stratum2_b200.scenegen import box_scene, cutout_scene, terrain_scene  # noqa: E402

GOLDEN_SEED = 1_000_000  # frame seeds of the oracle images; GPU tests use seeds < 100000


def box_case():
    wl = box_scene(seed=1, width=64, height=64)
    p = _abi.S2RenderParams()
    p.min_path_length, p.max_path_length = 2, 5
    p.flags = _abi.FLAG_LAMBERTIAN | _abi.FLAG_PIXEL_JITTER
    p.environment_sample_probability = 0.9
    p.restir_candidates = 32
    return wl, p


def terrain_case():
    wl = terrain_scene(seed=2, grid=128, spheres=8, sphere_level=2, width=64, height=36, tiles=2, area_lights=2,
                         sun_radiance=50.0, sun_cone_degrees=5.0)
    p = _abi.S2RenderParams()
    p.min_path_length, p.max_path_length = 1, 6
    p.flags = _abi.FLAG_PIXEL_JITTER
    p.environment_sample_probability = 0.9
    p.restir_candidates = 32
    return wl, p


def cutout_case():
    wl = cutout_scene(seed=3, width=64, height=64)
    p = _abi.S2RenderParams()
    p.min_path_length, p.max_path_length = 0, 5
    p.flags = _abi.FLAG_PIXEL_JITTER
    p.environment_sample_probability = 0.9
    p.restir_candidates = 32
    return wl, p


def cfg2_case():
    """The benchmark workload (1920x1080 terrain, 5e3 sun, path length 3..12, pixel centres) on
    the pixel subset x = 15 + 30 i, y = 15 + 30 j (64 x 36 pixels)."""
    wl = terrain_scene(seed=2)
    p = _abi.S2RenderParams()
    p.min_path_length, p.max_path_length = 3, 12
    p.flags = 0
    p.environment_sample_probability = 0.9
    p.restir_candidates = 32
    return wl, p


def cfg5_case():
    """The learned-cache workload: the benchmark terrain with 8 area lights (1920x1080, 5e3 sun,
    path length 3..12, pixel centres), on the same pixel subset as cfg2_case."""
    wl = terrain_scene(seed=2, area_lights=8)
    p = _abi.S2RenderParams()
    p.min_path_length, p.max_path_length = 3, 12
    p.flags = 0
    p.environment_sample_probability = 0.9
    p.restir_candidates = 32
    return wl, p


SUBSET = {"cfg2_1920x1080_subset30": ((15, 15, 1920, 1080), 30), "cfg5_1920x1080_subset30": ((15, 15, 1920, 1080), 30)}
CASES = {"box_64x64": (box_case, 16384), "terrain_64x36": (terrain_case, 131072), "cutout_64x64": (cutout_case, 16384),
         "cfg2_1920x1080_subset30": (cfg2_case, 262144), "cfg5_1920x1080_subset30": (cfg5_case, 262144)}


def make(name: str, out_dir: Path = HERE):
    fn, spp = CASES[name]
    wl, p = fn()
    p.spp = spp
    p.frame_seed = GOLDEN_SEED
    osc = OracleScene(wl.scene, 1)
    t = time.time()
    if name in SUBSET:
        rect, stride = SUBSET[name]
        r = osc.render(wl.view, p, wl.width, wl.height, precision=64, rect=rect, stride=stride)
        sel = (slice(rect[1], rect[3], stride), slice(rect[0], rect[2], stride))
        np.savez_compressed(out_dir / f"{name}_fp64_{spp}spp.npz", mean=r["mean"][sel].astype(np.float32),
                            var_of_mean=r["var_of_mean"][sel].astype(np.float32), spp=spp, seed=GOLDEN_SEED,
                            rect=np.array(rect), stride=stride)
    else:
        r = osc.render(wl.view, p, wl.width, wl.height, precision=64)
        np.savez_compressed(out_dir / f"{name}_fp64_{spp}spp.npz", mean=r["mean"].astype(np.float32),
                            var_of_mean=r["var_of_mean"].astype(np.float32), spp=spp, seed=GOLDEN_SEED)
    print(name, f"{time.time() - t:.1f}s", float(r["mean"].mean()))


if __name__ == "__main__":
    for n in (sys.argv[1:] or CASES):
        make(n)
