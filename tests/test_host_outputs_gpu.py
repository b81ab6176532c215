"""Host outputs of s2_render: the first-hit AOVs are copied on a side stream while the later
bounces render, and page-locked frame buffers (Device.host_result(pinned=True)) are reused in place.
Every output must equal the device-buffer render of the same call bit for bit, in one wave and
across several waves."""
import ctypes as C

import numpy as np
import pytest

from stratum2_b200 import _abi
from stratum2_b200.api import Device
from stratum2_b200.scenegen import box_scene

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("wave_paths", [0, 4096 * 3])
def test_host_outputs_equal_device_outputs(device, wave_paths):
    import torch
    W = H = 64
    wl = box_scene(seed=1, width=W, height=H)
    device.upload_scene(wl.scene)
    p = Device.default_params()
    p.spp, p.min_path_length, p.max_path_length, p.frame_seed = 16, 2, 5, 77
    p.flags = _abi.FLAG_LAMBERTIAN | _abi.FLAG_PIXEL_JITTER
    p.wave_paths = wave_paths
    fresh = device.render(wl.view, W, H, params=p)
    pinned = Device.host_result(W, H, pinned=True)
    again = device.render(wl.view, W, H, params=p, out=pinned)
    assert again is pinned
    t = {k: torch.zeros((H, W, c), dtype=dt, device="cuda") for k, c, dt in
         (("radiance", 4, torch.float32), ("albedo", 4, torch.float32), ("visibility", 2, torch.int32),
          ("depth", 4, torch.float32), ("prev_uv", 2, torch.float32), ("ids32", 2, torch.int32))}
    aov = _abi.S2Aovs(*(t[k].data_ptr() for k in ("radiance", "albedo", "visibility", "depth", "prev_uv", "ids32")))
    device.render_device(wl.view, p, aov)
    torch.cuda.synchronize()
    for k in t:
        d = t[k].cpu().numpy()
        if d.dtype == np.int32:
            d = d.view(np.uint32)
        np.testing.assert_array_equal(getattr(fresh, k), d, err_msg=k)
        np.testing.assert_array_equal(getattr(pinned, k), d, err_msg=k)
    assert fresh.stats.extension_rays == pinned.stats.extension_rays > 0
    with pytest.raises(ValueError):
        device.render(wl.view, W + 1, H, params=p, out=pinned)
