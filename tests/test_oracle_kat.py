"""Known-answer tests that pin the oracle: RNG, packing, half floats, BSDF normalisation and
reciprocity, and a white-furnace render with a closed-form answer."""
import ctypes as C

import numpy as np
import pytest

from oracle_lib import OracleScene, oracle
from stratum2_b200 import _abi
from stratum2_b200.scene import Material, Scene, make_view


def pcg4d_numpy(v):
    """Independent restatement of pcg4d (src/Shaders/common/rng.hlsli:23-35)."""
    v = v.astype(np.uint32).copy()
    with np.errstate(over="ignore"):
        v = v * np.uint32(1664525) + np.uint32(1013904223)
        x, y, z, w = v.T.copy()
        x += y * w; y += z * x; z += x * y; w += y * z
        x ^= x >> np.uint32(16); y ^= y >> np.uint32(16); z ^= z >> np.uint32(16); w ^= w >> np.uint32(16)
        x += y * w; y += z * x; z += x * y; w += y * z
    return np.stack([x, y, z, w], 1)


def test_pcg4d_matches_independent_restatement():
    rng = np.random.default_rng(0)
    v = rng.integers(0, 2 ** 32, (1000, 4), dtype=np.uint64).astype(np.uint32)
    out = np.zeros_like(v)
    oracle().oracle_pcg4d(v.ctypes.data, out.ctypes.data, len(v))
    np.testing.assert_array_equal(out, pcg4d_numpy(v))
    # first draw of pixel (0,0), seed 0: counter 1
    out1 = np.zeros((1, 4), np.uint32)
    oracle().oracle_pcg4d(np.array([[0, 0, 0, 1]], np.uint32).ctypes.data, out1.ctypes.data, 1)
    np.testing.assert_array_equal(out1, pcg4d_numpy(np.array([[0, 0, 0, 1]], np.uint32)))


def test_half_round_matches_numpy_float16():
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.normal(0, 1, 2000), rng.uniform(0, 7e4, 2000), 10 ** rng.uniform(-9, 5, 2000)]).astype(np.float32)
    ref = x.astype(np.float16).astype(np.float32)
    mine = np.array([oracle().oracle_half_round(float(v)) for v in x], np.float32)
    np.testing.assert_array_equal(mine, ref)


def test_octahedral_normal_round_trip():
    rng = np.random.default_rng(2)
    v = rng.normal(size=(2000, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    out = np.zeros(3)
    worst = 0.0
    for n in v:
        p = oracle().oracle_pack_normal(*n)
        oracle().oracle_unpack_normal(p, out.ctypes.data)
        worst = max(worst, float(np.arccos(np.clip(out @ n, -1, 1))))
    assert worst < 1e-4  # 16-bit SNORM octahedral quantization


def _mat_words(m: Material):
    w, _ = m.packed_words()
    return np.array(w, np.uint32)


def _eval(words, lam, win, wout):
    res = np.zeros(5)
    oracle().oracle_bsdf_eval(words.ctypes.data, C.c_float(0), int(lam), np.asarray(win, np.float64).ctypes.data,
                              np.asarray(wout, np.float64).ctypes.data, res.ctypes.data)
    return res


def _sample(words, lam, win, rnd):
    res = np.zeros(10)
    oracle().oracle_bsdf_sample(words.ctypes.data, int(lam), np.asarray(win, np.float64).ctypes.data,
                                np.asarray(rnd, np.float64).ctypes.data, res.ctypes.data)
    return res


MATERIALS = [
    (Material(base_color=(0.6, 0.5, 0.4)), True),
    (Material.metallic_roughness((0.8, 0.3, 0.2), 0.5, 0.0), False),
    (Material.metallic_roughness((0.9, 0.9, 0.9), 0.35, 1.0), False),
    (Material.metallic_roughness((0.2, 0.7, 0.3), 0.9, 0.0), False),
]


@pytest.mark.parametrize("mi", range(len(MATERIALS)))
def test_bsdf_pdf_integrates_to_at_most_one(mi):
    """Monte Carlo integral of evalPdf over the upper hemisphere (uniform directions) <= 1.
    (For directions below an opaque surface the reference's evalPdf returns the unscaled lobe
    probabilities, disney.hlsli:212-228; f is 0 there, so that value only multiplies zero.)"""
    m, lam = MATERIALS[mi]
    words = _mat_words(m)
    rng = np.random.default_rng(3)
    win = np.array([0.3, -0.2, 0.9])
    win /= np.linalg.norm(win)
    n = 40000
    d = rng.normal(size=(n, 3))
    d[:, 2] = np.abs(d[:, 2])
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pdf = np.array([_eval(words, lam, win, o)[3] for o in d])
    integral = pdf.mean() * 2 * np.pi
    assert integral <= 1.03
    if lam:
        assert abs(integral - 1) < 0.03


@pytest.mark.parametrize("mi", range(len(MATERIALS)))
def test_bsdf_reciprocity(mi):
    """f(in,out)/|out.z| == f(out,in)/|in.z| for the reflection lobes (Lambert, Disney opaque)."""
    m, lam = MATERIALS[mi]
    words = _mat_words(m)
    rng = np.random.default_rng(4)
    for _ in range(200):
        a = rng.normal(size=3); a[2] = abs(a[2]) + 0.05; a /= np.linalg.norm(a)
        b = rng.normal(size=3); b[2] = abs(b[2]) + 0.05; b /= np.linalg.norm(b)
        f1 = _eval(words, lam, a, b)[:3] / abs(b[2])
        f2 = _eval(words, lam, b, a)[:3] / abs(a[2])
        np.testing.assert_allclose(f1, f2, rtol=2e-2, atol=1e-6)  # Disney's diffuse retro term is near-reciprocal


@pytest.mark.parametrize("mi", range(len(MATERIALS)))
def test_bsdf_sample_estimates_reflectance(mi):
    """E[f/pdf] over sampled directions == integral of f over the hemisphere (estimated with
    uniform directions): sampling and evaluation agree."""
    m, lam = MATERIALS[mi]
    words = _mat_words(m)
    rng = np.random.default_rng(5)
    win = np.array([0.2, 0.1, 0.97]); win /= np.linalg.norm(win)
    n = 20000
    est = np.zeros(3)
    for r in rng.uniform(size=(n, 3)):
        s = _sample(words, lam, win, r)
        if s[9] and s[6] > 0:
            est += s[3:6] / s[6]
    est /= n
    d = rng.normal(size=(n, 3)); d /= np.linalg.norm(d, axis=1, keepdims=True)
    ref = np.mean([_eval(words, lam, win, o)[:3] for o in d], 0) * 4 * np.pi
    np.testing.assert_allclose(est, ref, rtol=0.06, atol=2e-3)


def furnace_scene(albedo: float, emission: float):
    """Closed cube [-1,1]^3 of 12 inward-facing emissive Lambertian triangles."""
    s = Scene()
    m = s.add_material(Material(base_color=(albedo,) * 3, emission=(emission,) * 3))
    faces = [
        ((-1, -1, -1), (-1, -1, 1), (1, -1, 1), (1, -1, -1)),
        ((-1, 1, -1), (1, 1, -1), (1, 1, 1), (-1, 1, 1)),
        ((-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1)),
        ((-1, -1, 1), (-1, 1, 1), (1, 1, 1), (1, -1, 1)),
        ((-1, -1, -1), (-1, 1, -1), (-1, 1, 1), (-1, -1, 1)),
        ((1, -1, -1), (1, -1, 1), (1, 1, 1), (1, 1, -1)),
    ]
    for f in faces:
        s.add_instance(s.add_mesh(np.array(f, np.float32), np.array([[0, 1, 2], [0, 2, 3]])), m)
    return s


@pytest.mark.parametrize("min_len,max_len", [(0, 4), (2, 5)])
def test_white_furnace_closed_form(min_len, max_len):
    """Radiance seen inside a closed emissive Lambertian box: Le * sum_{k=min..max} a^(k-1)
    (path length k = k segments; NEE + MIS + Russian roulette are unbiased for it)."""
    a = 0.5
    s = furnace_scene(a, 1.0)
    aq = 128 / 255  # 8-bit quantized albedo
    expected = sum(aq ** (k - 1) for k in range(max(min_len, 1), max_len + 1))
    osc = OracleScene(s, 1)
    view = make_view((0.1, -0.2, 0.05), 8, 8, 60.0)
    p = _abi.S2RenderParams()
    p.min_path_length, p.max_path_length, p.spp, p.frame_seed = min_len, max_len, 256, 0
    p.flags = _abi.FLAG_LAMBERTIAN
    p.environment_sample_probability = 0.9
    out = osc.render(view, p, 8, 8)
    mean = out["mean"].mean()
    se = np.sqrt(out["var_of_mean"].mean() / 64)
    assert abs(mean - expected) < 5 * se + 1e-3 * expected, (mean, expected, se)
