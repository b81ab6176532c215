"""Failure detection of the bounded device waits, on the GPU without a GPU fault.

The radiance cache's tensor-core kernels wait on mbarriers with an iteration limit; when a wait
gives up, the kernel records it in the context's status word, waits (bounded) for work in flight,
frees its TMEM and returns, and the host call reports S2_ERR_TIMEOUT.  s2_inject_wait_timeout makes
the next inference launch wait on a barrier that nothing will arrive on (the layer's MMA and commit
are not issued, so nothing is in flight) with a short poll limit.  The tests check the reported
status, and that the context stays usable: the next calls succeed and give the same results as
before the injection."""
import ctypes as C

import numpy as np
import pytest

from stratum2_b200 import Device, _abi
from stratum2_b200.scenegen import box_scene

pytestmark = pytest.mark.gpu
POLLS = 4096


def _cache_params():
    p = _abi.S2CacheParams()
    _abi.lib().s2_cache_default_params(p)
    for k in range(3):
        p.box_min[k], p.box_max[k] = -1.0, 1.0
    return p


def test_cache_query_wait_timeout_is_reported_and_the_context_recovers(device):
    lib = _abi.lib()
    device.cache_init(_cache_params())
    pos = np.random.default_rng(0).uniform(-1, 1, (5000, 3)).astype(np.float32)
    before = device.cache_query(pos)
    assert lib.s2_inject_wait_timeout(device._h, POLLS) == _abi.S2_OK
    with pytest.raises(_abi.S2Error) as e:
        device.cache_query(pos)
    assert e.value.code == _abi.S2_ERR_TIMEOUT
    assert b"timed out" in lib.s2_last_error(device._h)
    after = device.cache_query(pos)  # one-shot: the next launch runs normally, TMEM was released
    np.testing.assert_array_equal(after, before)


def test_render_cache_step_wait_timeout_is_reported_and_the_next_render_succeeds(device):
    lib = _abi.lib()
    wl = box_scene(seed=1, n_random=100, width=32, height=32)
    device.upload_scene(wl.scene)
    device.cache_init()
    p = _abi.S2RenderParams()
    lib.s2_default_render_params(p)
    p.spp, p.min_path_length, p.max_path_length, p.frame_seed = 2, 2, 5, 3
    p.flags = _abi.FLAG_LAMBERTIAN | _abi.FLAG_RADIANCE_CACHE
    p.cache_bounces, p.cache_train_paths = 1, 256
    device.render(wl.view, wl.width, wl.height, params=p)
    assert lib.s2_inject_wait_timeout(device._h, POLLS) == _abi.S2_OK
    with pytest.raises(_abi.S2Error) as e:
        device.render(wl.view, wl.width, wl.height, params=p)
    assert e.value.code == _abi.S2_ERR_TIMEOUT
    r = device.render(wl.view, wl.width, wl.height, params=p)
    assert np.isfinite(r.radiance).all() and r.radiance[..., :3].sum() > 0


def test_injection_arguments_are_checked():
    lib = _abi.lib()
    d = Device(0)
    try:
        assert lib.s2_inject_wait_timeout(d._h, POLLS) == _abi.S2_ERR_NO_SCENE  # no cache yet
        d.cache_init(_cache_params())
        assert lib.s2_inject_wait_timeout(d._h, 0) == _abi.S2_ERR_INVALID
        assert lib.s2_inject_wait_timeout(d._h, (1 << 20) + 1) == _abi.S2_ERR_INVALID
    finally:
        d.close()
