"""Autotuner persistence (CPU) and the tuning entry points (GPU)."""
import numpy as np
import pytest

from stratum2_b200 import _abi, autotune


def test_tuning_json_round_trip(tmp_path):
    t = _abi.S2Tuning()
    t.wave_paths, t.trav_tris_per_step, t.trav_vote8, t.refill_min, t.shade_order = 1 << 23, 2, 5, 12, 1
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


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [_abi.FLAG_LAMBERTIAN, 0, _abi.FLAG_RESTIR_DI])
def test_queue_orders_keep_the_image_bitwise(device, flags):
    """Sorting paths by material before shading, and continuation rays by origin cell and octant
    before tracing, only reorders the queue: each path keeps its own random state and accumulator
    slot, so the image is bit-identical in every order, also across several waves (wave_paths
    below the path count) and in the batched streaming entry point."""
    from stratum2_b200.scenegen import textured_box_scene
    wl = textured_box_scene(seed=4, width=48, height=48, spheres=3)
    device.upload_scene(wl.scene)
    p = device.default_params()
    p.spp, p.min_path_length, p.max_path_length, p.flags, p.frame_seed = 8, 2, 6, flags | _abi.FLAG_PIXEL_JITTER, 11
    p.restir_candidates = 4
    queue = _abi.S2Tuning()
    queue.shade_order = _abi.SHADE_ORDER_QUEUE
    device.set_tuning(queue)
    ref = device.render(wl.view, 48, 48, params=p).radiance
    for wave in (0, 4096):
        for trace in (_abi.TRACE_ORDER_QUEUE, _abi.TRACE_ORDER_COHERENT):
            t = _abi.S2Tuning()
            t.wave_paths, t.trace_order = wave, trace
            device.set_tuning(t)
            out = device.render(wl.view, 48, 48, params=p).radiance
            np.testing.assert_array_equal(out, ref)
    # batched streaming: fixed-point accumulation, so also independent of the shading order
    device.set_tuning(queue)
    a, _ = device.render_views([wl.view], p)
    device.set_tuning(None)
    b, _ = device.render_views([wl.view], p)
    np.testing.assert_array_equal(a[0].radiance, b[0].radiance)
    device.set_tuning(None)


@pytest.mark.gpu
@pytest.mark.parametrize("scene,flags", [("textured_box", _abi.FLAG_LAMBERTIAN), ("textured_box", 0),
                                         ("terrain", 0), ("terrain", _abi.FLAG_RESTIR_DI)])
def test_shading_records_keep_the_image_bitwise(device, scene, flags):
    """The baked per-triangle shading records (S2Tuning.shade_records, on by default) hold
    make_shading's own per-triangle terms: images and first-hit AOVs are bit-identical to the
    gather through instance, vertex info, indices and positions, on meshes with texture
    coordinates (not baked: the textured walls) and without (baked: spheres, terrain)."""
    from stratum2_b200.scenegen import terrain_scene, textured_box_scene
    wl = textured_box_scene(seed=4, width=48, height=48, spheres=3) if scene == "textured_box" else \
        terrain_scene(seed=2, grid=128, spheres=8, sphere_level=2, width=64, height=36, tiles=2, area_lights=2)
    device.upload_scene(wl.scene)
    p = device.default_params()
    p.spp, p.min_path_length, p.max_path_length, p.flags, p.frame_seed = 8, 1, 6, flags | _abi.FLAG_PIXEL_JITTER, 17
    p.restir_candidates = 4
    off = _abi.S2Tuning()
    off.shade_records = _abi.SHADE_RECORDS_OFF
    device.set_tuning(off)
    ref = device.render(wl.view, wl.width, wl.height, params=p)
    device.set_tuning(None)
    out = device.render(wl.view, wl.width, wl.height, params=p)
    np.testing.assert_array_equal(out.radiance, ref.radiance)
    np.testing.assert_array_equal(out.albedo, ref.albedo)
    np.testing.assert_array_equal(out.visibility, ref.visibility)
    np.testing.assert_array_equal(out.depth, ref.depth)


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [_abi.FLAG_LAMBERTIAN, 0, _abi.FLAG_RESTIR_DI])
def test_shadow_merge_keeps_the_image_bitwise(device, flags):
    """Tracing a bounce's shadow rays in the next bounce's traversal launch (S2Tuning.shadow_merge,
    on by default) instead of a launch of their own changes when they are traced, not what they
    add: every contribution still reaches its accumulator slot before the next shade, so images,
    AOVs and ray counts are bit-identical, in one wave and in several."""
    from stratum2_b200.scenegen import terrain_scene
    wl = terrain_scene(seed=2, grid=128, spheres=8, sphere_level=2, width=64, height=36, tiles=2, area_lights=2)
    device.upload_scene(wl.scene)
    p = device.default_params()
    p.spp, p.min_path_length, p.max_path_length, p.flags, p.frame_seed = 8, 1, 7, flags | _abi.FLAG_PIXEL_JITTER, 23
    p.restir_candidates = 4
    for wave in (0, 4096):
        off = _abi.S2Tuning()
        off.wave_paths, off.shadow_merge = wave, _abi.SHADOW_MERGE_OFF
        device.set_tuning(off)
        ref = device.render(wl.view, wl.width, wl.height, params=p)
        on = _abi.S2Tuning()
        on.wave_paths = wave
        device.set_tuning(on)
        out = device.render(wl.view, wl.width, wl.height, params=p)
        np.testing.assert_array_equal(out.radiance, ref.radiance)
        np.testing.assert_array_equal(out.albedo, ref.albedo)
        assert out.stats.extension_rays == ref.stats.extension_rays
        assert out.stats.shadow_rays == ref.stats.shadow_rays > 0
        assert out.stats.kernel_launches < ref.stats.kernel_launches
    # the batched streaming form: fixed-point pixel totals, so also bit-identical
    off = _abi.S2Tuning()
    off.shadow_merge = _abi.SHADOW_MERGE_OFF
    device.set_tuning(off)
    a, sa = device.render_views([wl.view, wl.view], p)
    device.set_tuning(None)
    b, sb = device.render_views([wl.view, wl.view], p)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x.radiance, y.radiance)
    assert sa.shadow_rays == sb.shadow_rays > 0 and sa.extension_rays == sb.extension_rays
    device.set_tuning(None)


@pytest.mark.gpu
def test_pixel_centre_hint_keeps_the_hits(device):
    """Renders of 8 or more samples per pixel test each camera ray first against the triangle its
    pixel's centre ray hits.  The closest hit (ties to the lowest instance and primitive) does not
    depend on the order triangles are found, so an 8-spp render in two waves of 4 (hinted) equals
    two progressive 4-spp calls (no hint): the same AOVs bit for bit and the same radiance."""
    from stratum2_b200.scenegen import terrain_scene
    wl = terrain_scene(seed=2, grid=128, spheres=8, sphere_level=2, width=64, height=36, tiles=2, area_lights=2)
    device.upload_scene(wl.scene)
    p = device.default_params()
    p.spp, p.min_path_length, p.max_path_length, p.flags, p.frame_seed = 8, 1, 6, _abi.FLAG_PIXEL_JITTER, 31
    p.wave_paths = 4 * wl.width * wl.height
    hinted = device.render(wl.view, wl.width, wl.height, params=p)
    p.spp, p.wave_paths = 4, 0
    first = device.render(wl.view, wl.width, wl.height, params=p)
    p.flags |= _abi.FLAG_ACCUMULATE
    p.frame_seed = 31 + 4     # sample k of a frame draws from frame_seed + k
    acc = device.render(wl.view, wl.width, wl.height, params=p)
    for name in ("ids32", "visibility", "depth", "albedo"):
        np.testing.assert_array_equal(getattr(first, name), getattr(hinted, name))
    np.testing.assert_allclose(acc.radiance, hinted.radiance, rtol=1e-6, atol=1e-7)
