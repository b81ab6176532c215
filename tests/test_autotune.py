"""Autotuner persistence (CPU) and the tuning entry points (GPU)."""
import numpy as np
import pytest

from stratum2_b200 import _abi, autotune


def test_tuning_json_round_trip(tmp_path):
    t = _abi.S2Tuning()
    t.wave_paths, t.trav_tris_per_step, t.trav_vote8, t.refill_min = 1 << 23, 2, 5, 12
    table = {"gpu|tris=10|64x64|spp=4|len=2-5|flags=0": autotune.to_dict(t)}
    autotune.save(table, tmp_path / "t.json")
    back = autotune.load(tmp_path / "t.json")
    assert back == table
    assert autotune.to_dict(autotune.from_dict(back[next(iter(back))])) == autotune.to_dict(t)
    assert autotune.load(tmp_path / "missing.json") == {}


@pytest.mark.gpu
def test_autotune_applies_a_tuning_that_keeps_the_image(device, tmp_path):
    from stratum2_b200.scenegen import box_scene
    wl = box_scene(seed=1, width=64, height=64)
    device.upload_scene(wl.scene)
    p = device.default_params()
    p.spp, p.min_path_length, p.max_path_length, p.flags, p.frame_seed = 8, 2, 5, _abi.FLAG_LAMBERTIAN, 3
    device.set_tuning(None)
    ref = device.render(wl.view, 64, 64, params=p).radiance
    res = autotune.autotune(device, wl.view, p, path=tmp_path / "tune.json")
    assert res["searched"] and res["trials"] > 10
    t = device.get_tuning()
    assert autotune.to_dict(t) == res["tuning"]
    tuned = device.render(wl.view, 64, 64, params=p).radiance
    np.testing.assert_allclose(tuned, ref, rtol=1e-5, atol=1e-6)
    again = autotune.autotune(device, wl.view, p, path=tmp_path / "tune.json")
    assert not again["searched"] and again["tuning"] == res["tuning"]
    bad = _abi.S2Tuning()
    bad.trav_vote8 = 12
    with pytest.raises(_abi.S2Error):
        device.set_tuning(bad)
    device.set_tuning(None)
