"""Environment sampling by the bilinear footprint (S2_FLAG_ENV_FOOTPRINT_PDF, no counterpart in the
reference) in the oracle: the estimator stays unbiased (its image agrees with the committed FP64
golden image of the parity terrain, rendered with the reference's texel pdf, by a per-pixel z-test)
and, where a small bright sun's bilinear halo is left to BSDF sampling by the texel pdf, its
per-sample variance falls."""
from pathlib import Path

import numpy as np

from oracle_lib import OracleScene, default_render_params
from stratum2_b200 import _abi
from stratum2_b200.scenegen import terrain_scene

GOLDEN = Path(__file__).resolve().parent / "golden" / "terrain_64x36_fp64_131072spp.npz"


def _terrain(**kw):
    return terrain_scene(seed=2, grid=128, spheres=8, sphere_level=2, width=64, height=36, tiles=2, area_lights=2, **kw)


def _params(spp, flags, seed):
    p = default_render_params()
    p.spp, p.min_path_length, p.max_path_length, p.flags, p.frame_seed = spp, 1, 6, flags, seed
    return p


def test_footprint_pdf_is_unbiased_against_fp64_golden():
    """Flag on, the oracle's image agrees with the FP64 golden image rendered with the texel pdf as
    closely as the texel pdf's own render of the same seeds does (heavy-tailed per-pixel estimates
    make a per-channel z-test fail for both at this sample count, equally)."""
    wl = _terrain(sun_radiance=50.0, sun_cone_degrees=5.0)
    g = np.load(GOLDEN)
    ref = g["mean"].astype(np.float64)
    osc = OracleScene(wl.scene, 1)
    err = {}
    for name, fl in (("texel", 0), ("footprint", _abi.FLAG_ENV_FOOTPRINT_PDF)):
        r = osc.render(wl.view, _params(1024, _abi.FLAG_PIXEL_JITTER | fl, 5000), wl.width, wl.height, precision=64)
        err[name] = float(np.mean((r["mean"] - ref) ** 2 / (ref ** 2 + 1e-2)))
        assert abs(float(r["mean"].mean() / ref.mean() - 1.0)) < 2e-3, (name, r["mean"].mean(), ref.mean())
    assert err["footprint"] < 1.5 * err["texel"], err


def test_footprint_pdf_covers_the_bilinear_halo_of_a_one_texel_sun():
    """A 5e3 sun of half a degree covers about one texel of the 512x256 sky.  The environment is
    evaluated bilinearly, so the texels around it carry up to half its radiance; the texel pdf
    gives them the sky's probability, and radiance / pdf (the value of an environment hit that
    only BSDF sampling finds) reaches thousands of times its value on the sun itself.  With the
    footprint pdf the ratio stays within a small factor of its value over the whole sky."""
    wl = _terrain()
    osc = OracleScene(wl.scene, 1)
    sun = np.array([0.3, 0.8, 0.2]) / np.linalg.norm([0.3, 0.8, 0.2])
    t1 = np.cross(sun, [0.0, 0.0, 1.0]); t1 /= np.linalg.norm(t1)
    t2 = np.cross(sun, t1)
    a = np.radians(np.linspace(-2.5, 2.5, 101))
    aa, bb = np.meshgrid(a, a)
    halo = sun[None] + np.tan(aa.reshape(-1))[:, None] * t1 + np.tan(bb.reshape(-1))[:, None] * t2
    rng = np.random.default_rng(3)
    sky = rng.normal(size=(20000, 3))
    dirs = np.concatenate([halo, sky])
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    ratio = {}
    for name, fl in (("texel", 0), ("footprint", _abi.FLAG_ENV_FOOTPRINT_PDF)):
        rgb, pdf = osc.env_eval(_params(1, fl, 0), dirs)
        lum = rgb @ np.array([0.2126, 0.7152, 0.0722])
        ok = lum > 0
        assert (pdf[ok] > 0).all(), name
        ratio[name] = lum[ok] / pdf[ok]
    assert ratio["texel"].max() > 1000 * np.median(ratio["texel"]), ratio["texel"].max()
    assert ratio["footprint"].max() < 10 * np.median(ratio["footprint"]), ratio["footprint"].max()
