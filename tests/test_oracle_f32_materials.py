"""The oracle's f32-material mode (the differentiable renderer's materials): identical to the
reference's 8-bit materials where no texture modulates them, different where one does.  CPU only."""
import numpy as np

from oracle_lib import OracleScene
from stratum2_b200 import _abi
from stratum2_b200.scenegen import box_scene, textured_box_scene

ORACLE_F32 = 1 << 30


def params(flags):
    p = _abi.S2RenderParams()
    _abi.lib().s2_default_render_params(p)
    p.spp, p.flags, p.frame_seed, p.min_path_length, p.max_path_length = 2, flags, 3, 0, 4
    return p


def test_untextured_materials_are_unchanged():
    wl = box_scene(seed=1, width=24, height=24)
    osc = OracleScene(wl.scene, 1)
    a = osc.render(wl.view, params(_abi.FLAG_LAMBERTIAN), 24, 24)["mean"]
    b = osc.render(wl.view, params(_abi.FLAG_LAMBERTIAN | ORACLE_F32), 24, 24)["mean"]
    np.testing.assert_array_equal(a, b)


def test_textured_materials_differ_by_quantisation_only():
    wl = textured_box_scene(width=24, height=24)
    osc = OracleScene(wl.scene, 1)
    a = osc.render(wl.view, params(_abi.FLAG_LAMBERTIAN), 24, 24)["mean"]
    b = osc.render(wl.view, params(_abi.FLAG_LAMBERTIAN | ORACLE_F32), 24, 24)["mean"]
    assert not np.array_equal(a, b)
    assert np.abs(a - b).mean() < 0.02 * np.abs(a).mean()


def test_detached_sampling_with_the_same_textures_is_the_plain_estimator():
    import ctypes
    from oracle_lib import oracle
    L = oracle()
    L.oracle_scene_set_sampling.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    wl = textured_box_scene(width=24, height=24)
    a = OracleScene(wl.scene, 1)
    b = OracleScene(wl.scene, 1)
    ref = a.render(wl.view, params(ORACLE_F32), 24, 24)["mean"]
    L.oracle_scene_set_sampling(a.h, b.h)
    det = a.render(wl.view, params(ORACLE_F32), 24, 24)["mean"]
    L.oracle_scene_set_sampling(a.h, None)
    np.testing.assert_array_equal(ref, det)
