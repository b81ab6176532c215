"""Differentiable rendering (s2_render_diff) and the adjoint path replay (s2_render_adjoint).

* The differentiable forward is the wavefront renderer's estimator: the same random numbers per
  (pixel, sample) give the same samples (untextured scenes, where f32 and 8-bit materials agree), and
  on the textured box it matches the oracle's f32-material mode sample by sample.
* With sampling independent of the parameter (Lambertian BSDF and area-light NEE for albedo texels;
  BSDF sampling only for environment texels; no Russian roulette), the estimator of a fixed seed is a
  smooth function of the texels, and the adjoint must equal its central finite differences (common
  random numbers, eps 0.05 on one texel; the estimator is at most quadratic in one texel, where
  central differences are exact): within 1e-2 relative.  The FP64 oracle's finite differences of
  the same estimator give the reference gradient.
* Disney: roughness and base colour change the sampled directions, so the full estimator's finite
  differences are dominated by paths that jump across edges (their spread over seeds is tens of times
  the gradient).  The adjoint's estimator holds sampling fixed; the FP64 oracle's detached-sampling
  mode (sampling from the unperturbed textures, BSDF values from the perturbed ones) has exactly
  that estimator, and its central differences must match the adjoint within 2e-2.
* torch.autograd: the bridge returns the adjoint's gradients, and Adam on an L2 image loss (4 spp per
  step; residual and adjoint from independent renders) brings the image of a perturbed albedo
  texture back toward the target image.
"""
import ctypes

import numpy as np
import pytest

from oracle_lib import OracleScene, oracle
from stratum2_b200 import _abi
from stratum2_b200.scenegen import textured_box_scene
from test_render_gpu import box_wl, terrain_wl

pytestmark = pytest.mark.gpu
J, LAM = _abi.FLAG_PIXEL_JITTER, _abi.FLAG_LAMBERTIAN
NO_RR, NO_NEE = _abi.FLAG_NO_RR, _abi.FLAG_NO_NEE
ORACLE_F32 = 1 << 30  # the oracle's f32-material mode (the differentiable renderer's materials)


def params(spp, flags, seed=0, minl=0, maxl=4):
    p = _abi.S2RenderParams()
    _abi.lib().s2_default_render_params(p)
    p.spp, p.flags, p.frame_seed, p.min_path_length, p.max_path_length = spp, flags, seed, minl, maxl
    return p


def diverging(a, b):
    return float(np.mean((np.abs(a[..., :3] - b[..., :3]) > 1e-3 * np.abs(b[..., :3]) + 1e-4).any(-1)))


@pytest.fixture(scope="module")
def tbox(device):
    wl = textured_box_scene()
    device.upload_scene(wl.scene)
    return wl


@pytest.mark.parametrize("scene", ["box", "terrain"])
def test_diff_forward_is_the_wavefront_estimator(device, scene):
    wl = box_wl() if scene == "box" else terrain_wl()
    flags, minl, maxl = (LAM | J, 2, 5) if scene == "box" else (J, 1, 6)
    device.upload_scene(wl.scene)
    bad = 0.0
    for k in range(8):
        p = params(1, flags, seed=100 + k, minl=minl, maxl=maxl)
        a, st = device.render_diff(wl.view, wl.width, wl.height, p)
        b = device.render(wl.view, wl.width, wl.height, params=p).radiance
        bad += diverging(a, b) / 8
        assert st.extension_rays > 0
    assert bad <= 0.01, bad


@pytest.mark.parametrize("flags", [LAM | J, J])
def test_diff_forward_matches_oracle_f32_materials(device, tbox, flags):
    wl = tbox
    device.upload_scene(wl.scene)
    osc = OracleScene(wl.scene, 1)
    bad = 0.0
    for k in range(8):
        p = params(1, flags, seed=200 + k)
        a, _ = device.render_diff(wl.view, wl.width, wl.height, p)
        po = params(1, flags | ORACLE_F32, seed=200 + k)
        o = osc.render(wl.view, po, wl.width, wl.height)["mean"]
        bad += diverging(a, np.concatenate([o, np.ones(o.shape[:2] + (1,))], -1)) / 8
    assert bad <= 0.01, bad


def loss(device, wl, p, d):
    img, _ = device.render_diff(wl.view, wl.width, wl.height, p)
    return float(np.sum(d[..., :3].astype(np.float64) * img[..., :3]))


def fd_check(device, wl, p, image, channels, eps, n=48, seed=0):
    rng = np.random.default_rng(seed)
    d = rng.uniform(0, 1, (wl.height, wl.width, 4)).astype(np.float32)
    g = device.render_adjoint(wl.view, p, d, images=[image])[image]
    base = wl.scene.images[image].copy()
    mag = np.abs(g[..., channels]).max(-1)
    flat = np.argsort(mag.ravel())[::-1]
    picks = list(flat[:n // 2]) + list(rng.choice(flat[:max(n, int((mag > 0).sum()))], n // 2, replace=False))
    errs = []
    try:
        for f in picks:
            y, x = divmod(int(f), base.shape[1])
            c = channels[int(np.argmax(np.abs(g[y, x, channels])))]
            t = base.copy()
            t[y, x, c] += eps
            device.update_image(image, t)
            lp = loss(device, wl, p, d)
            t[y, x, c] -= 2 * eps
            device.update_image(image, t)
            lm = loss(device, wl, p, d)
            fd = (lp - lm) / (2 * eps)
            errs.append(abs(fd - g[y, x, c]) / (abs(fd) + 1e-3 * np.abs(g[..., channels]).max()))
    finally:
        device.update_image(image, base)
    return np.array(errs), g, d


def test_albedo_gradient_equals_finite_differences(device, tbox):
    wl = tbox
    device.upload_scene(wl.scene)
    errs, _, _ = fd_check(device, wl, params(4, LAM | NO_RR | J, seed=7), 0, [0, 1, 2], 0.05)
    assert np.max(errs) < 1e-2, np.sort(errs)[-5:]


def test_environment_gradient_equals_finite_differences(device, tbox):
    wl = tbox
    device.upload_scene(wl.scene)
    errs, _, _ = fd_check(device, wl, params(4, LAM | NO_RR | NO_NEE | J, seed=8), 2, [0, 1, 2], 0.05)
    assert np.max(errs) < 1e-2, np.sort(errs)[-5:]


def test_albedo_gradient_matches_fp64_oracle(device, tbox):
    """The FP64 oracle's central differences of the same estimator (f32-material mode, same seeds)."""
    wl = tbox
    device.upload_scene(wl.scene)
    p = params(2, LAM | NO_RR | J, seed=9)
    rng = np.random.default_rng(3)
    d = rng.uniform(0, 1, (wl.height, wl.width, 4)).astype(np.float32)
    g = device.render_adjoint(wl.view, p, d, images=[0])[0]
    base = wl.scene.images[0].copy()
    order = np.argsort(np.abs(g[..., :3]).max(-1).ravel())[::-1][:8]
    po = params(2, LAM | NO_RR | J | ORACLE_F32, seed=9)
    try:
        for f in order:
            y, x = divmod(int(f), base.shape[1])
            c = int(np.argmax(np.abs(g[y, x, :3])))
            vals = []
            for sgn in (1, -1):
                wl.scene.images[0] = base.copy()
                wl.scene.images[0][y, x, c] += sgn * 0.05
                o = OracleScene(wl.scene, 1).render(wl.view, po, wl.width, wl.height)["mean"]
                vals.append(np.sum(d[..., :3] * o))
            fd = (vals[0] - vals[1]) / 0.1
            assert abs(fd - g[y, x, c]) <= 1e-2 * abs(fd) + 1e-4 * np.abs(g).max(), (y, x, c, fd, g[y, x, c])
    finally:
        wl.scene.images[0] = base


def detached_fd(wl, p, image, ch, eps, texel=None):
    """FP64 oracle central difference of sum(image) under detached sampling: image `image` channel
    `ch` shifted by +-eps (all texels, or one texel (y, x)) for evaluation only."""
    L = oracle()
    L.oracle_scene_set_sampling.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    base = wl.scene.images[image].copy()
    samp = OracleScene(wl.scene, 1)
    vals = []
    try:
        for sgn in (1, -1):
            t = base.copy()
            if texel is None:
                t[..., ch] += sgn * eps
            else:
                t[texel[0], texel[1], ch] += sgn * eps
            wl.scene.images[image] = t
            ev = OracleScene(wl.scene, 1)
            L.oracle_scene_set_sampling(ev.h, samp.h)
            vals.append(ev.render(wl.view, p, wl.width, wl.height)["mean"].sum())
            L.oracle_scene_set_sampling(ev.h, None)
    finally:
        wl.scene.images[image] = base
    return (vals[0] - vals[1]) / (2 * eps)


@pytest.mark.parametrize("image,ch", [(1, 1), (0, 0)])
def test_disney_gradients_match_detached_oracle(device, tbox, image, ch):
    wl = tbox
    device.upload_scene(wl.scene)
    p = params(4, J, seed=31)
    po = params(4, J | ORACLE_F32, seed=31)
    d = np.ones((wl.height, wl.width, 4), np.float32)
    g = device.render_adjoint(wl.view, p, d, images=[image])[image][..., ch]
    fd = detached_fd(wl, po, image, ch, 1e-3)
    assert abs(g.sum() - fd) <= 2e-2 * abs(fd), (g.sum(), fd)
    for f in np.argsort(np.abs(g).ravel())[::-1][:4]:
        y, x = divmod(int(f), g.shape[1])
        fdt = detached_fd(wl, po, image, ch, 1e-3, texel=(y, x))
        assert abs(g[y, x] - fdt) <= 2e-2 * abs(fdt) + 1e-3 * np.abs(g).max(), (y, x, g[y, x], fdt)


def test_torch_autograd_bridge_and_inverse_rendering(device, tbox):
    torch = pytest.importorskip("torch")
    from stratum2_b200.autograd import render

    wl = tbox
    device.upload_scene(wl.scene)
    true = torch.tensor(wl.scene.images[0], device="cuda")
    p = params(4, LAM | J, seed=21)
    # the bridge's gradient is the adjoint's
    tex = true.clone().requires_grad_(True)
    img = render(device, wl.view, wl.width, wl.height, p, {0: tex})
    w = torch.rand_like(img)
    (img * w).sum().backward()
    ref = device.render_adjoint(wl.view, p, w.detach().cpu().numpy(), images=[0])[0][..., :3]
    np.testing.assert_allclose(tex.grad.cpu().numpy(), ref, rtol=1e-5, atol=1e-6)
    # inverse rendering: recover an 8 x 8 albedo texture from a target image
    wl8 = textured_box_scene(tex_res=8)
    device.upload_scene(wl8.scene)
    true8 = torch.tensor(wl8.scene.images[0], device="cuda")
    target = render(device, wl8.view, wl8.width, wl8.height, params(256, LAM | J, seed=5), {0: true8}).detach()

    def image_error(t):  # 256-spp image of texture t against the target, common seeds
        with torch.no_grad():
            img = render(device, wl8.view, wl8.width, wl8.height, params(256, LAM | J, seed=77), {0: t})
            return ((img - target)[..., :3] ** 2).mean().item()

    gen = torch.Generator(device="cuda").manual_seed(0)
    x = (true8 + 0.2 * torch.randn(true8.shape, generator=gen, device="cuda")).clamp(0.05, 1.0).requires_grad_(True)
    opt = torch.optim.Adam([x], lr=0.02)
    floor = image_error(true8)
    err0, tex0 = image_error(x.detach()), ((x.detach() - true8) ** 2).mean().item()
    SPP = 16
    for it in range(60):
        opt.zero_grad()
        # decorrelated gradient of the L2 loss: the residual from one render, the adjoint from a render
        # with other seeds (one set of samples for both would bias the gradient toward lower variance;
        # sample s of a call uses seed frame_seed + s, so the two renders take disjoint seed blocks)
        with torch.no_grad():
            a = render(device, wl8.view, wl8.width, wl8.height, params(SPP, LAM | J, seed=100000 + 2 * SPP * it), {0: x})
        b = render(device, wl8.view, wl8.width, wl8.height, params(SPP, LAM | J, seed=100000 + 2 * SPP * it + SPP), {0: x})
        (2 * (a - target).detach() * b)[..., :3].mean().backward()
        opt.step()
        with torch.no_grad():
            x.clamp_(0.0, 1.0)
    err1, tex1 = image_error(x.detach()), ((x.detach() - true8) ** 2).mean().item()
    device.upload_scene(wl.scene)
    assert tex1 < 0.25 * tex0, (tex0, tex1)
    assert err1 - floor < 0.5 * (err0 - floor), (floor, err0, err1)
