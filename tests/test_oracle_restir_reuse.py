"""The oracle's restatement of the ReSTIR DI hash-grid reuse (testrenderer.slang:608-726,
hashgrid.hlsli:14-119) converges to the FP64 golden image (plain NEE) on a pixel subset of the
box scene, and the first call of a reuse sequence (no previous grid) is the RIS-only render.
CPU only."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from oracle_lib import OracleScene, oracle
from stratum2_b200 import _abi
from stratum2_b200.scenegen import box_scene

GOLDEN = Path(__file__).resolve().parent / "golden"
FLAGS = _abi.FLAG_LAMBERTIAN | _abi.FLAG_PIXEL_JITTER | _abi.FLAG_RESTIR_DI


def params(seed, flags, m=4):
    p = _abi.S2RenderParams()
    p.min_path_length, p.max_path_length, p.spp, p.frame_seed, p.flags = 2, MAXLEN, 1, seed, flags
    p.environment_sample_probability = 0.9
    p.restir_candidates = m
    p.restir_max_m = 3.0
    p.restir_grid_cells = 100000
    p.restir_grid_cell_size = 0.5
    return p


MAXLEN = 5
M32 = 0xFFFFFFFF


def pcg_py(v):
    st = (v * 747796405 + 2891336453) & M32
    w = (((st >> ((st >> 28) + 4)) ^ st) * 277803737) & M32
    return (w >> 22) ^ w


def xxhash32_py(p):
    h = (p + 374761393) & M32
    h = (668265263 * (((h << 17) | (h >> 15)) & M32)) & M32
    h = (2246822519 * (h ^ (h >> 15))) & M32
    h = (3266489917 * (h ^ (h >> 13))) & M32
    return h ^ (h >> 16)


def test_hash_functions_known_answers():
    # pcg (Jarzynski & Olano 2020) and the one-word xxhash32 (rng.hlsli:5-22), the hash-grid keys
    L = oracle()
    L.oracle_pcg_hash.restype = L.oracle_xxhash32.restype = C.c_uint32
    L.oracle_pcg_hash.argtypes = L.oracle_xxhash32.argtypes = [C.c_uint32]
    assert L.oracle_pcg_hash(0) == pcg_py(0) == 129708002
    assert L.oracle_xxhash32(0) == xxhash32_py(0) == 878055299
    for v in np.random.default_rng(0).integers(0, 2**32, 200, dtype=np.uint64).tolist() + [M32, 1, 2**31]:
        assert L.oracle_pcg_hash(v) == pcg_py(v)
        assert L.oracle_xxhash32(v) == xxhash32_py(v)


@pytest.fixture(scope="module")
def box():
    wl = box_scene(seed=1, width=64, height=64)
    return wl, OracleScene(wl.scene, 1)


def test_first_reuse_call_is_ris(box):
    wl, osc = box
    rect = (0, 0, 64, 64)
    # a call without reuse drops any previous grid; the first reuse call then has nothing to reuse
    osc.render(wl.view, params(1, FLAGS), 64, 64, rect=rect, stride=8)
    a = osc.render(wl.view, params(2, FLAGS | _abi.FLAG_RESTIR_REUSE), 64, 64, rect=rect, stride=8)["mean"]
    b = osc.render(wl.view, params(2, FLAGS), 64, 64, rect=rect, stride=8)["mean"]
    np.testing.assert_array_equal(a, b)
    # the second reuse call reuses the first one's reservoirs and differs
    osc.render(wl.view, params(2, FLAGS | _abi.FLAG_RESTIR_REUSE), 64, 64, rect=rect, stride=8)
    c = osc.render(wl.view, params(3, FLAGS | _abi.FLAG_RESTIR_REUSE), 64, 64, rect=rect, stride=8)["mean"]
    d = osc.render(wl.view, params(3, FLAGS), 64, 64, rect=rect, stride=8)["mean"]
    assert not np.array_equal(c, d)


def test_oracle_reuse_converges_to_nee(box):
    """Paths of up to 3 segments (NEE at the first two vertices, where the reuse acts): 16 batches
    of 128 reuse frames against 32768-spp plain NEE on every 4th pixel in x and y."""
    wl, osc = box
    global MAXLEN
    MAXLEN = 3
    try:
        stride, nb, frames = 4, 16, 128
        sel = (slice(0, 64, stride), slice(0, 64, stride))
        p = params(900000, _abi.FLAG_LAMBERTIAN | _abi.FLAG_PIXEL_JITTER)
        p.spp = 32768
        ref = osc.render(wl.view, p, 64, 64, stride=stride)
        means = []
        seed = 50000
        for b in range(nb):
            acc = 0.0
            for f in range(frames):
                r = osc.render(wl.view, params(seed, FLAGS | _abi.FLAG_RESTIR_REUSE), 64, 64, stride=stride)
                acc = acc + r["mean"][sel]
                seed += 1
            means.append(acc / frames)
    finally:
        MAXLEN = 5
    means = np.stack(means)
    m, v = means.mean(0), means.var(0, ddof=1) / nb
    gm, gv = ref["mean"][sel], ref["var_of_mean"][sel]
    z = (m - gm) / np.sqrt(v + gv + (1e-5 * np.abs(gm) + 1e-9) ** 2)
    assert np.mean(np.abs(z) > 5) <= 0.01, np.sort(np.abs(z).ravel())[-5:]
    assert abs(z.mean()) < 0.25, z.mean()


def test_oracle_reuse_visibility_first_call_and_second_call(box):
    """gReSTIR_DI_Reuse_Visibility (testrenderer.slang:611-616, 689-694, 742-743) in the oracle:
    without a previous grid the traced visibility changes nothing (an occluded canonical sample
    contributes zero either way), so the first call equals plain reuse's bit for bit; with a grid
    the reused samples differ."""
    wl, osc = box
    rect = (0, 0, 64, 64)
    V = _abi.FLAG_RESTIR_REUSE_VISIBILITY
    osc.render(wl.view, params(1, FLAGS), 64, 64, rect=rect, stride=8)
    a = osc.render(wl.view, params(2, FLAGS | _abi.FLAG_RESTIR_REUSE), 64, 64, rect=rect, stride=8)["mean"]
    osc.render(wl.view, params(1, FLAGS), 64, 64, rect=rect, stride=8)
    b = osc.render(wl.view, params(2, FLAGS | _abi.FLAG_RESTIR_REUSE | V), 64, 64, rect=rect, stride=8)["mean"]
    np.testing.assert_array_equal(a, b)
    c = osc.render(wl.view, params(3, FLAGS | _abi.FLAG_RESTIR_REUSE | V), 64, 64, rect=rect, stride=8)["mean"]
    osc.render(wl.view, params(1, FLAGS), 64, 64, rect=rect, stride=8)
    osc.render(wl.view, params(2, FLAGS | _abi.FLAG_RESTIR_REUSE), 64, 64, rect=rect, stride=8)
    d = osc.render(wl.view, params(3, FLAGS | _abi.FLAG_RESTIR_REUSE), 64, 64, rect=rect, stride=8)["mean"]
    assert np.isfinite(c).all() and not np.array_equal(c, d)
