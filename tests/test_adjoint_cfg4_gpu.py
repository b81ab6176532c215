"""The adjoint path replay at the inverse-rendering workload's specification: the box with 200
level-3 icospheres (256,012 triangles), a 1024^2 RGB albedo map, a 1024^2 roughness map and a 256x128
environment map, rendered here at 128x128 (the workload renders 512x512; the gradients are the same
estimator, a quarter of the pixels keeps the finite differences affordable), 4 spp, path length up
to 4.  Gradients of L = sum(d * image) with random weights d:

* albedo (image 0) and environment (image 2) texels: central finite differences with eps 1e-3 of
  the same estimator (common random numbers; sampling independent of these texels: Lambertian BSDF
  with area-light NEE for albedo, BSDF sampling only for the environment, no Russian roulette) on
  64 random interior texels that the paths reach, within 1e-2 relative (relative to |fd| plus 1e-3
  of the largest gradient, the float rounding floor of a one-texel change);
* roughness (image 1, channel y): the FP64 oracle's central differences (eps 1e-3) of the
  detached-sampling estimator (sampling from the unperturbed textures, BSDF values from the
  perturbed ones: the estimator the adjoint differentiates), on 8 random interior texels the paths
  reach, within 1e-2."""
import numpy as np
import pytest

from stratum2_b200 import _abi
from stratum2_b200.scenegen import textured_box_scene
from test_adjoint_gpu import ORACLE_F32, detached_fd, loss, params

pytestmark = pytest.mark.gpu
J, LAM = _abi.FLAG_PIXEL_JITTER, _abi.FLAG_LAMBERTIAN
NO_RR, NO_NEE = _abi.FLAG_NO_RR, _abi.FLAG_NO_NEE
EPS = 1e-3


@pytest.fixture(scope="module")
def cfg4(device):
    wl = textured_box_scene(n_random=0, width=128, height=128, tex_res=1024, env_res=(256, 128), spheres=200,
                            sphere_level=3)
    device.upload_scene(wl.scene)
    assert device.bvh_stats.triangle_count == 256_012
    return wl


def _interior_reached(g, channels, n, rng):
    mag = np.abs(g[..., channels]).max(-1)
    mag[0, :] = mag[-1, :] = 0
    mag[:, 0] = mag[:, -1] = 0
    cand = np.flatnonzero(mag.ravel() > 1e-4 * mag.max())
    assert len(cand) >= n, len(cand)
    return rng.choice(cand, n, replace=False)


@pytest.mark.parametrize("image,flags", [(0, LAM | NO_RR | J), (2, LAM | NO_RR | NO_NEE | J)], ids=["albedo", "environment"])
def test_cfg4_gradient_equals_central_differences(device, cfg4, image, flags):
    wl = cfg4
    device.upload_scene(wl.scene)
    rng = np.random.default_rng(40 + image)
    p = params(4, flags, seed=41 + image)
    d = rng.uniform(0, 1, (wl.height, wl.width, 4)).astype(np.float32)
    g = device.render_adjoint(wl.view, p, d, images=[image])[image]
    base = wl.scene.images[image].copy()
    gmax = np.abs(g[..., :3]).max()
    errs = []
    try:
        for f in _interior_reached(g, [0, 1, 2], 64, rng):
            y, x = divmod(int(f), base.shape[1])
            c = int(np.argmax(np.abs(g[y, x, :3])))
            t = base.copy()
            t[y, x, c] += EPS
            device.update_image(image, t)
            lp = loss(device, wl, p, d)
            t[y, x, c] -= 2 * EPS
            device.update_image(image, t)
            lm = loss(device, wl, p, d)
            fd = (lp - lm) / (2 * EPS)
            errs.append(abs(fd - g[y, x, c]) / (abs(fd) + 1e-3 * gmax))
    finally:
        device.update_image(image, base)
    errs = np.array(errs)
    assert errs.max() < 1e-2, np.sort(errs)[-5:]


def test_cfg4_roughness_gradient_matches_detached_fp64_oracle(device, cfg4):
    wl = cfg4
    device.upload_scene(wl.scene)
    rng = np.random.default_rng(44)
    p = params(4, J, seed=45)
    po = params(4, J | ORACLE_F32, seed=45)
    d = np.ones((wl.height, wl.width, 4), np.float32)
    g = device.render_adjoint(wl.view, p, d, images=[1])[1][..., 1]
    gmax = np.abs(g).max()
    for f in _interior_reached(g[..., None], [0], 8, rng):
        y, x = divmod(int(f), g.shape[1])
        fdt = detached_fd(wl, po, 1, 1, EPS, texel=(y, x))
        assert abs(g[y, x] - fdt) <= 1e-2 * abs(fdt) + 1e-3 * gmax, (y, x, g[y, x], fdt)
