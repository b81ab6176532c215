"""The glTF texture repack on the GPU (s2_repack_metallic_roughness, the reference's from_gltf_pbr
pass, convert_material.slang:33-69) against the oracle's float64 restatement (oracle/gltf_oracle.py),
bit for bit, for every 8-bit value and every combination of present sources; and a loaded glTF
scene rendered on the GPU against the FP64 oracle at the same seed and converged."""
import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle_lib import OracleScene
from stratum2_b200 import _abi
from stratum2_b200.gltf import load_gltf
from test_gltf import _document
from test_render_gpu import assert_converged, assert_same_seed, batches, make_params

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
from gltf_oracle import repack_metallic_roughness as oracle_repack  # noqa: E402

pytestmark = pytest.mark.gpu


def _sources(h, w, seed):
    rng = np.random.default_rng(seed)
    base = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    flat = np.arange(h * w * 4) % 256  # every 8-bit value in every channel
    base.reshape(-1)[:] = flat.astype(np.uint8)
    mr = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    em = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    em[0, :3, :3] = 0        # black emission texels: 0/0 saturates to 0
    em[1, 0, :3] = (255, 7, 7)
    return base, mr, em


def _assert_same(got, want):
    gi, ga, gm = got
    wi, wa, wm = want
    for k in range(4):
        np.testing.assert_array_equal(gi[k].view(np.uint32), wi[k].view(np.uint32), err_msg=f"packed[{k}]")
    if wa is None:
        assert ga is None
    else:
        np.testing.assert_array_equal(ga.view(np.uint32), wa.view(np.uint32))
    assert gm == wm


@pytest.mark.parametrize("present", [(1, 1, 1), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (0, 1, 1)])
def test_repack_matches_oracle_bitwise(device, present):
    base, mr, em = _sources(37, 53, 11)  # odd extent: a partial last block
    src = [t if p else None for t, p in zip((base, mr, em), present)]
    _assert_same(device.repack_metallic_roughness(*src), oracle_repack(*src))


def test_repack_opaque_base_reports_255(device):
    base, _, _ = _sources(8, 8, 2)
    base[..., 3] = 255
    imgs, alpha, min_alpha = device.repack_metallic_roughness(base, None, None)
    assert min_alpha == 255 and (alpha == 1.0).all()


def test_repack_device_pointers(device):
    """on_device = 1: sources and outputs in device memory (torch tensors), the same bits."""
    import torch
    base, mr, em = _sources(64, 96, 5)
    h, w = base.shape[:2]
    dev = [torch.from_numpy(t).cuda() for t in (base, mr, em)]
    outs = [torch.empty((h, w, 4), dtype=torch.float32, device="cuda") for _ in range(4)]
    alpha = torch.empty((h, w), dtype=torch.float32, device="cuda")
    ptrs = (C.c_void_p * 4)(*[o.data_ptr() for o in outs])
    min_alpha = C.c_uint32(0)
    torch.cuda.synchronize()
    rc = _abi.lib().s2_repack_metallic_roughness(device._h, w, h, *[t.data_ptr() for t in dev], ptrs,
                                                 alpha.data_ptr(), C.byref(min_alpha), 1)
    assert rc == _abi.S2_OK
    got = ([o.cpu().numpy() for o in outs], alpha.cpu().numpy(), int(min_alpha.value))
    _assert_same(got, oracle_repack(base, mr, em))


def test_repack_rejects_bad_arguments(device):
    base, _, _ = _sources(4, 4, 1)
    lib = _abi.lib()
    imgs = [np.empty((4, 4, 4), np.float32) for _ in range(4)]
    ptrs = (C.c_void_p * 4)(*[im.ctypes.data for im in imgs])
    m = C.c_uint32(0)
    assert lib.s2_repack_metallic_roughness(device._h, 4, 4, None, None, None, ptrs, None, C.byref(m), 0) == _abi.S2_ERR_INVALID
    assert lib.s2_repack_metallic_roughness(device._h, 0, 4, base.ctypes.data, None, None, ptrs, None, C.byref(m), 0) == _abi.S2_ERR_INVALID
    alpha = np.empty((4, 4), np.float32)
    assert lib.s2_repack_metallic_roughness(device._h, 4, 4, None, base.ctypes.data, None, ptrs, alpha.ctypes.data,
                                            C.byref(m), 0) == _abi.S2_ERR_INVALID


class _Workload:
    def __init__(self, g, width, height):
        self.scene, self.view, self.width, self.height = g.scene, g.views[0], width, height


@pytest.fixture(scope="module")
def gltf_wl(device, tmp_path_factory):
    """The test document (textured, alpha-masked, emissive quad and a transmissive triangle under a
    node hierarchy, a camera looking down onto them) loaded through the GPU repack, under a uniform
    environment."""
    tmp = tmp_path_factory.mktemp("gltf")
    doc, *_ = _document(np.random.default_rng(0))
    (tmp / "s.gltf").write_text(json.dumps(doc))
    g = load_gltf(tmp / "s.gltf", width=64, height=48, device=device)
    g.scene.set_environment((1.0, 1.0, 1.0))
    wl = _Workload(g, 64, 48)
    device.upload_scene(wl.scene)
    return wl, OracleScene(wl.scene, 1)


def test_gltf_loaded_through_the_gpu_repack_equals_the_oracle_repack(device, tmp_path):
    doc, *_ = _document(np.random.default_rng(0))
    (tmp_path / "s.gltf").write_text(json.dumps(doc))
    a = load_gltf(tmp_path / "s.gltf", device=device)
    b = load_gltf(tmp_path / "s.gltf", repack=oracle_repack)
    assert bytes(a.scene.material_data) == bytes(b.scene.material_data)
    assert len(a.scene.images) == len(b.scene.images)
    for x, y in zip(a.scene.images, b.scene.images):
        np.testing.assert_array_equal(np.asarray(x).view(np.uint32), np.asarray(y).view(np.uint32))


@pytest.mark.parametrize("extra", [_abi.FLAG_PIXEL_JITTER, _abi.FLAG_LAMBERTIAN | _abi.FLAG_PIXEL_JITTER])
def test_gltf_render_same_seed_matches_fp64_oracle(device, gltf_wl, extra):
    wl, osc = gltf_wl
    device.upload_scene(wl.scene)
    p = make_params(1, 0, 4, extra, seed=21)
    assert_same_seed(device, osc, wl, p, f"glTF flags {extra}")
    r = device.render(wl.view, wl.width, wl.height, params=p)
    assert r.stats.nan_count == 0
    assert (r.ids32[..., 0] != 0xFFFFFFFF).any()


def test_gltf_render_converges_to_the_oracle(device, gltf_wl):
    wl, osc = gltf_wl
    device.upload_scene(wl.scene)
    p = make_params(1, 0, 4, _abi.FLAG_PIXEL_JITTER, seed=0)
    g_mean, g_var = batches(device, wl, p, 8, 128, 1000)
    p.spp, p.frame_seed = 1024, 77
    o = osc.render(wl.view, p, wl.width, wl.height)
    assert_converged(g_mean, g_var, o["mean"], o["var_of_mean"], 1e-2, "glTF scene")
