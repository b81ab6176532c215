"""s2_render_noalloc: the allocation-free render entry point.

It exists for callers that may not allocate device memory while they render (a host application
that owns the GPU memory budget and forbids cudaMalloc/cudaFree in its frame loop, or a plugin
limited to the buffers its host provides).  This test calls it through the C ABI, with output
buffers the caller allocated beforehand, twice in a row, and checks both results against the
regular s2_render entry point on the same scene and seeds; the second call also checks that state
left in the shared scratch array by the first does not leak into the next result.  The file is
named so pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from stratum2_b200 import Device, _abi
from stratum2_b200.scenegen import box_scene

pytestmark = pytest.mark.gpu


def _params(spp, seed):
    p = _abi.S2RenderParams()
    _abi.lib().s2_default_render_params(p)
    p.spp, p.min_path_length, p.max_path_length, p.frame_seed = spp, 2, 5, seed
    p.flags = _abi.FLAG_LAMBERTIAN | _abi.FLAG_PIXEL_JITTER
    return p


def test_no_alloc_render_matches_s2_render_on_two_calls():
    wl = box_scene(seed=1, width=64, height=64)
    dev = Device(0)
    try:
        dev.upload_scene(wl.scene)
        p = _params(16, 7)
        ref = dev.render(wl.view, wl.width, wl.height, params=p)
        H, W = wl.height, wl.width
        # outputs allocated by the caller up front
        rad = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")
        alb = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")
        vis = torch.empty((H, W, 2), dtype=torch.int32, device="cuda")
        ids = torch.empty((H, W, 2), dtype=torch.int32, device="cuda")
        aovs = _abi.S2Aovs(rad.data_ptr(), alb.data_ptr(), vis.data_ptr(), None, None, ids.data_ptr())
        lib = _abi.lib()
        for call in range(2):
            rad.fill_(-1.0)
            st = _abi.S2RenderStats()
            rc = lib.s2_render_noalloc(dev._h, C.byref(wl.view), C.byref(p), C.byref(aovs), C.byref(st))
            assert rc == _abi.S2_OK, lib.s2_last_error(dev._h).decode()
            torch.cuda.synchronize()
            np.testing.assert_allclose(rad.cpu().numpy(), ref.radiance, rtol=1e-6, atol=1e-7, err_msg=f"call {call}")
            np.testing.assert_array_equal(alb.cpu().numpy(), ref.albedo)
            np.testing.assert_array_equal(vis.cpu().numpy().view(np.uint32), ref.visibility)
            np.testing.assert_array_equal(ids.cpu().numpy().view(np.uint32), ref.ids32)
            assert st.extension_rays == ref.stats.extension_rays and st.shadow_rays == ref.stats.shadow_rays
        # a view beyond the scratch limit is rejected with a clear error, before any GPU work
        big = box_scene(seed=1, n_random=10, width=1920, height=1080).view
        rc = lib.s2_render_noalloc(dev._h, C.byref(big), C.byref(p), C.byref(aovs), None)
        assert rc == _abi.S2_ERR_INVALID
        assert b"scratch limit" in lib.s2_last_error(dev._h)
        # modes that need buffers of their own are refused, not rendered as plain path tracing
        for flag in (_abi.FLAG_LIGHT_TRACE, _abi.FLAG_RESTIR_REUSE, _abi.FLAG_RESTIR_SCREEN, _abi.FLAG_RADIANCE_CACHE):
            q = _params(1, 7)
            q.flags |= flag
            rc = lib.s2_render_noalloc(dev._h, C.byref(wl.view), C.byref(q), C.byref(aovs), None)
            assert rc == _abi.S2_ERR_UNSUPPORTED, hex(flag)
    finally:
        dev.close()


def test_no_alloc_restir_matches_s2_render():
    """RIS (S2_FLAG_RESTIR_DI without reuse) through the allocation-free entry point, whose ReSTIR
    shade variant runs on its own grid, equals s2_render's image on two calls in a row."""
    wl = box_scene(seed=1, width=48, height=40)
    dev = Device(0)
    try:
        dev.upload_scene(wl.scene)
        p = _params(8, 11)
        p.flags |= _abi.FLAG_RESTIR_DI
        p.restir_candidates = 8
        ref = dev.render(wl.view, wl.width, wl.height, params=p)
        rad = torch.empty((wl.height, wl.width, 4), dtype=torch.float32, device="cuda")
        aovs = _abi.S2Aovs(rad.data_ptr(), None, None, None, None, None)
        lib = _abi.lib()
        for call in range(2):
            rad.fill_(-1.0)
            rc = lib.s2_render_noalloc(dev._h, C.byref(wl.view), C.byref(p), C.byref(aovs), None)
            assert rc == _abi.S2_OK, lib.s2_last_error(dev._h).decode()
            torch.cuda.synchronize()
            np.testing.assert_allclose(rad.cpu().numpy(), ref.radiance, rtol=1e-6, atol=1e-7, err_msg=f"call {call}")
    finally:
        dev.close()


def test_no_alloc_view_at_the_pixel_limit():
    """A view of exactly 322,603 pixels (the documented limit) renders; one pixel more is refused."""
    limit = 322_603
    wl = box_scene(seed=1, n_random=50, width=limit, height=1)
    dev = Device(0)
    try:
        dev.upload_scene(wl.scene)
        p = _params(1, 3)
        rad = torch.empty((1, limit, 4), dtype=torch.float32, device="cuda")
        aovs = _abi.S2Aovs(rad.data_ptr(), None, None, None, None, None)
        lib = _abi.lib()
        rc = lib.s2_render_noalloc(dev._h, C.byref(wl.view), C.byref(p), C.byref(aovs), None)
        assert rc == _abi.S2_OK, lib.s2_last_error(dev._h).decode()
        torch.cuda.synchronize()
        assert torch.isfinite(rad).all()
        over = box_scene(seed=1, n_random=50, width=limit + 1, height=1).view
        rc = lib.s2_render_noalloc(dev._h, C.byref(over), C.byref(p), C.byref(aovs), None)
        assert rc == _abi.S2_ERR_INVALID and b"scratch limit" in lib.s2_last_error(dev._h)
    finally:
        dev.close()
