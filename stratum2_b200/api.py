"""Host-side mirror of the reference's renderer interface over the C ABI.

`Device` owns one S2Context (one CUDA stream).  `Device.render(...)` plays the role of
TestRenderer::render (src/App/TestRenderer.cpp:284-763) with the VCM path-length arguments
(--minPathLength / --maxPathLength, src/App/VCM.cpp:39-40) and the tonemapper's --exposure
(src/App/Tonemapper.cpp:25).  Errors raise S2Error with the library's message, matching the
reference's host-side exceptions (std::runtime_error).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import S2Error


@dataclass
class RenderResult:
    radiance: np.ndarray      # (H, W, 4) float32
    albedo: np.ndarray        # (H, W, 4) float32
    visibility: np.ndarray    # (H, W, 2) uint32
    depth: np.ndarray         # (H, W, 4) float32
    prev_uv: np.ndarray       # (H, W, 2) float32
    ids32: np.ndarray         # (H, W, 2) uint32
    stats: _abi.S2RenderStats


def rays_array(origins, directions, tmin=0.0, tmax=np.inf) -> np.ndarray:
    """Packs rays as S2Ray records (float32 x 8)."""
    o = np.asarray(origins, np.float32).reshape(-1, 3)
    d = np.asarray(directions, np.float32).reshape(-1, 3)
    n = o.shape[0]
    r = np.empty((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = tmin
    r[:, 4:7] = d
    r[:, 7] = tmax
    return r


def hits_from_bytes(buf: np.ndarray) -> dict:
    rec = np.frombuffer(buf.tobytes(), dtype=np.dtype([("t", "<f4"), ("instance", "<u4"), ("primitive", "<u4"),
                                                       ("b1", "<f4"), ("b2", "<f4")]))
    return {k: rec[k].copy() for k in rec.dtype.names}


class Device:
    def __init__(self, device: int = 0):
        self._lib = _abi.lib()
        h = C.c_void_p()
        rc = self._lib.s2_create(device, C.byref(h))
        if rc != _abi.S2_OK:
            raise S2Error(rc, "s2_create failed (no CUDA device?)")
        self._h = h
        self.bvh_stats = None
        self.scene = None

    def close(self):
        if self._h:
            self._lib.s2_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != _abi.S2_OK:
            raise S2Error(rc, self._lib.s2_last_error(self._h).decode())

    def upload_scene(self, scene, build: bool = True, max_leaf_size: int = 3, collapse: int = _abi.BVH_COLLAPSE_SAH):
        self.scene = scene
        d = scene.desc()
        self._check(self._lib.s2_scene_upload(self._h, C.byref(d)))
        if build:
            p = _abi.S2BvhParams(max_leaf_size=max_leaf_size, sah_bins=32, threads=0, collapse=collapse)
            st = _abi.S2BvhStats()
            self._check(self._lib.s2_build_bvh(self._h, C.byref(p), C.byref(st)))
            self.bvh_stats = st
        return self

    def trace(self, rays: np.ndarray, anyhit: bool = False, counted: bool = False):
        """Closest-hit (or first-hit) query for host rays (n x 8 float32, S2Ray layout)."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        out = np.zeros(n * 5, np.uint32)
        if counted:
            cnt = np.zeros(2 * n, np.uint32)
            self._check(self._lib.s2_trace_counted(self._h, rays.ctypes.data, n, int(anyhit), out.ctypes.data,
                                                   cnt.ctypes.data, 0))
            return hits_from_bytes(out), cnt.reshape(n, 2)
        self._check(self._lib.s2_trace(self._h, rays.ctypes.data, n, int(anyhit), out.ctypes.data, 0))
        return hits_from_bytes(out)

    def get_bvh(self):
        """The built BVH8 as host arrays: nodes (n, 128) uint8 and triangle records (m, 12) float32
        (layouts in csrc/s2_bvh.h)."""
        counts = np.zeros(2, np.uint64)
        self._check(self._lib.s2_get_bvh(self._h, None, None, counts.ctypes.data))
        nodes = np.zeros((int(counts[0]), 128), np.uint8)
        tris = np.zeros((int(counts[1]), 12), np.float32)
        self._check(self._lib.s2_get_bvh(self._h, nodes.ctypes.data, tris.ctypes.data, counts.ctypes.data))
        return nodes, tris

    def trace_device(self, rays_ptr: int, n: int, hits_ptr: int, anyhit: bool = False):
        """Same query with device pointers (e.g. torch tensors' data_ptr())."""
        self._check(self._lib.s2_trace(self._h, C.c_void_p(rays_ptr), n, int(anyhit), C.c_void_p(hits_ptr), 1))

    def set_stream(self, stream_ptr: int | None):
        self._check(self._lib.s2_set_stream(self._h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def sync(self):
        self._check(self._lib.s2_sync(self._h))

    @staticmethod
    def default_params() -> _abi.S2RenderParams:
        p = _abi.S2RenderParams()
        _abi.lib().s2_default_render_params(C.byref(p))
        return p

    @staticmethod
    def host_result(width: int, height: int, pinned: bool = False) -> RenderResult:
        """Host arrays for every output of one view, to pass as render(out=...) frame after frame.
        pinned=True page-locks them (through torch), so the library's device-to-host copies run
        asynchronously at full link speed and overlap the render."""
        def arr(shape, dt):
            if not pinned:
                return np.zeros(shape, dt)
            import torch
            t = torch.zeros(shape, dtype=torch.float32 if dt == np.float32 else torch.int32, pin_memory=True)
            return t.numpy().view(dt)  # the array keeps the pinned tensor alive
        return RenderResult(arr((height, width, 4), np.float32), arr((height, width, 4), np.float32),
                            arr((height, width, 2), np.uint32), arr((height, width, 4), np.float32),
                            arr((height, width, 2), np.float32), arr((height, width, 2), np.uint32),
                            _abi.S2RenderStats())

    def render(self, view: _abi.S2View, width: int, height: int, spp: int = 1, min_path_length: int = 0,
               max_path_length: int = 5, exposure: float = 0.0, frame_seed: int = 0, flags: int = 0,
               params: _abi.S2RenderParams | None = None, out: RenderResult | None = None) -> RenderResult:
        """s2_render into host arrays: new ones, or `out` (from host_result) reused in place."""
        p = params if params is not None else self.default_params()
        if params is None:
            p.min_path_length = min_path_length
            p.max_path_length = max_path_length
            p.exposure = exposure
            p.spp = spp
            p.frame_seed = frame_seed
            p.flags = flags
        r = out if out is not None else self.host_result(width, height)
        for a, c in ((r.radiance, 4), (r.albedo, 4), (r.visibility, 2), (r.depth, 4), (r.prev_uv, 2), (r.ids32, 2)):
            if a.shape != (height, width, c) or not a.flags.c_contiguous:
                raise ValueError("output arrays do not match the view")
        aov = _abi.S2Aovs(r.radiance.ctypes.data, r.albedo.ctypes.data, r.visibility.ctypes.data, r.depth.ctypes.data,
                          r.prev_uv.ctypes.data, r.ids32.ctypes.data)
        st = _abi.S2RenderStats()
        self._check(self._lib.s2_render(self._h, C.byref(view), C.byref(p), C.byref(aov), 1, C.byref(st)))
        r.stats = st
        return r

    # ---- vertex connection and merging (the reference's VCM renderer)
    @staticmethod
    def default_vcm_params() -> _abi.S2VcmParams:
        p = _abi.S2VcmParams()
        _abi.lib().s2_default_vcm_params(C.byref(p))
        return p

    def render_vcm(self, view: _abi.S2View, width: int, height: int,
                   params: _abi.S2VcmParams | None = None) -> RenderResult:
        """s2_render_vcm: `params.iterations` light + camera passes of one view (host arrays)."""
        p = params if params is not None else self.default_vcm_params()
        rad = np.zeros((height, width, 4), np.float32)
        alb = np.zeros((height, width, 4), np.float32)
        vis = np.zeros((height, width, 2), np.uint32)
        dep = np.zeros((height, width, 4), np.float32)
        puv = np.zeros((height, width, 2), np.float32)
        ids = np.zeros((height, width, 2), np.uint32)
        aov = _abi.S2Aovs(rad.ctypes.data, alb.ctypes.data, vis.ctypes.data, dep.ctypes.data, puv.ctypes.data,
                          ids.ctypes.data)
        st = _abi.S2RenderStats()
        self._check(self._lib.s2_render_vcm(self._h, C.byref(view), C.byref(p), C.byref(aov), 1, C.byref(st)))
        return RenderResult(rad, alb, vis, dep, puv, ids, st)

    def render_views(self, views, params: _abi.S2RenderParams, aovs: bool = True):
        """Batched render of several views (any resolutions) in one call (s2_render_views).
        Returns one RenderResult per view (host arrays) and the call's statistics."""
        n = len(views)
        arr = (_abi.S2View * n)(*views)
        outs = (_abi.S2Aovs * n)()
        results = []
        for k, v in enumerate(views):
            w = v.image_max[0] - v.image_min[0]
            h = v.image_max[1] - v.image_min[1]
            rad = np.zeros((h, w, 4), np.float32)
            alb = np.zeros((h, w, 4), np.float32) if aovs else None
            vis = np.zeros((h, w, 2), np.uint32) if aovs else None
            dep = np.zeros((h, w, 4), np.float32) if aovs else None
            puv = np.zeros((h, w, 2), np.float32) if aovs else None
            ids = np.zeros((h, w, 2), np.uint32) if aovs else None
            ptr = lambda a: a.ctypes.data if a is not None else None
            outs[k] = _abi.S2Aovs(ptr(rad), ptr(alb), ptr(vis), ptr(dep), ptr(puv), ptr(ids))
            results.append((rad, alb, vis, dep, puv, ids))
        st = _abi.S2RenderStats()
        self._check(self._lib.s2_render_views(self._h, C.cast(arr, C.c_void_p), n, C.byref(params),
                                              C.cast(outs, C.c_void_p), 1, C.byref(st)))
        return [RenderResult(*r, st) for r in results], st

    def render_views_device(self, views, params: _abi.S2RenderParams, outs) -> _abi.S2RenderStats:
        """s2_render_views with caller-owned device AOV buffers (one S2Aovs per view)."""
        n = len(views)
        arr = (_abi.S2View * n)(*views)
        oarr = (_abi.S2Aovs * n)(*outs)
        st = _abi.S2RenderStats()
        self._check(self._lib.s2_render_views(self._h, C.cast(arr, C.c_void_p), n, C.byref(params),
                                              C.cast(oarr, C.c_void_p), 0, C.byref(st)))
        return st

    def render_device(self, view, params: _abi.S2RenderParams, aovs: _abi.S2Aovs) -> _abi.S2RenderStats:
        st = _abi.S2RenderStats()
        self._check(self._lib.s2_render(self._h, C.byref(view), C.byref(params), C.byref(aovs), 0, C.byref(st)))
        return st

    # ---- learned radiance cache
    @staticmethod
    def cache_default_params() -> _abi.S2CacheParams:
        p = _abi.S2CacheParams()
        _abi.lib().s2_cache_default_params(C.byref(p))
        return p

    def cache_init(self, params: _abi.S2CacheParams | None = None):
        self._check(self._lib.s2_cache_init(self._h, C.byref(params) if params is not None else None))
        self._cache_log2 = (params.log2_table if params is not None else self.cache_default_params().log2_table)

    def cache_get_params(self) -> tuple[np.ndarray, np.ndarray]:
        w = np.zeros(_abi.CACHE_WEIGHTS, np.float32)
        t = np.zeros((_abi.CACHE_LEVELS, 1 << self._cache_log2, 2), np.float32)
        self._check(self._lib.s2_cache_get_params(self._h, w.ctypes.data, t.ctypes.data))
        return w, t

    def cache_set_params(self, weights=None, table=None):
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        t = None if table is None else np.ascontiguousarray(table, np.float32)
        self._check(self._lib.s2_cache_set_params(self._h, None if w is None else w.ctypes.data,
                                                  None if t is None else t.ctypes.data))

    def cache_query(self, positions) -> np.ndarray:
        """Cache radiance at world-space positions (n x 3) -> (n x 3) float32."""
        p = np.zeros((len(positions), 4), np.float32)
        p[:, :3] = positions
        out = np.zeros((len(positions), 4), np.float32)
        self._check(self._lib.s2_cache_query(self._h, p.ctypes.data, len(p), out.ctypes.data, 0))
        return out[:, :3]

    @staticmethod
    def _records(positions, targets):
        p = np.zeros((len(positions), 4), np.float32)
        p[:, :3] = positions
        t = np.zeros((len(targets), 4), np.float32)
        t[:, :3] = np.asarray(targets)[:, :3]
        return p, t

    def cache_train(self, positions, targets) -> float:
        """One Adam step on the records; returns the mean loss before the step."""
        p, t = self._records(positions, targets)
        loss = C.c_float(0)
        self._check(self._lib.s2_cache_train(self._h, p.ctypes.data, t.ctypes.data, len(p), C.byref(loss), 0))
        return loss.value

    def cache_gradients(self, positions, targets):
        """(mean loss, d loss / d weights, d loss / d table) without an optimiser step."""
        p, t = self._records(positions, targets)
        gw = np.zeros(_abi.CACHE_WEIGHTS, np.float32)
        gt = np.zeros((_abi.CACHE_LEVELS, 1 << self._cache_log2, 2), np.float32)
        loss = C.c_float(0)
        self._check(self._lib.s2_cache_gradients(self._h, p.ctypes.data, t.ctypes.data, len(p), gw.ctypes.data,
                                                 gt.ctypes.data, C.byref(loss), 0))
        return loss.value, gw, gt

    # ---- textures and differentiable rendering
    def update_image(self, index: int, texels):
        """Replaces image `index`'s texels (numpy array on the host, or a torch CUDA tensor)."""
        if hasattr(texels, "data_ptr") and getattr(texels, "is_cuda", False):
            t = texels.contiguous()
            self._check(self._lib.s2_update_image(self._h, index, C.c_void_p(t.data_ptr()), 1))
            return
        a = np.ascontiguousarray(texels, np.float32)
        self._check(self._lib.s2_update_image(self._h, index, a.ctypes.data, 0))

    def repack_metallic_roughness(self, base=None, metallic_roughness=None, emission=None):
        """Texture repack of a glTF metallic-roughness material on the GPU
        (s2_repack_metallic_roughness): uint8 RGBA8 sources of one (h, w) extent, None for an absent
        one -> (the four packed images as float32 (h, w, 4), the base colour's alpha as float32 (h, w)
        or None without a base colour, the smallest 8-bit alpha below 255)."""
        src = [None if t is None else np.ascontiguousarray(t, np.uint8) for t in (base, metallic_roughness, emission)]
        shapes = {t.shape for t in src if t is not None}
        if not shapes:
            raise ValueError("at least one source texture is required")
        if len(shapes) != 1 or len(next(iter(shapes))) != 3 or next(iter(shapes))[2] != 4:
            raise ValueError(f"sources must be RGBA8 arrays of one extent, got {sorted(shapes)}")
        h, w, _ = next(iter(shapes))
        imgs = [np.empty((h, w, 4), np.float32) for _ in range(4)]
        alpha = np.empty((h, w), np.float32) if base is not None else None
        ptrs = (C.c_void_p * 4)(*[im.ctypes.data for im in imgs])
        min_alpha = C.c_uint32(0)
        self._check(self._lib.s2_repack_metallic_roughness(
            self._h, w, h, *[None if t is None else t.ctypes.data for t in src], ptrs,
            None if alpha is None else alpha.ctypes.data, C.byref(min_alpha), 0))
        return imgs, alpha, int(min_alpha.value)

    def render_diff(self, view, width: int, height: int, params: _abi.S2RenderParams):
        """Image of the differentiable renderer (f32 materials): (H, W, 4) float32 and statistics."""
        out = np.zeros((height, width, 4), np.float32)
        st = _abi.S2RenderStats()
        self._check(self._lib.s2_render_diff(self._h, C.byref(view), C.byref(params), out.ctypes.data, 1, C.byref(st)))
        return out, st

    def render_diff_device(self, view, params: _abi.S2RenderParams, out_ptr: int) -> _abi.S2RenderStats:
        st = _abi.S2RenderStats()
        self._check(self._lib.s2_render_diff(self._h, C.byref(view), C.byref(params), C.c_void_p(out_ptr), 0, C.byref(st)))
        return st

    def render_adjoint(self, view, params: _abi.S2RenderParams, d_image: np.ndarray, images=None):
        """Texel gradients of sum(d_image * render_diff(...)) for the images in `images` (default all):
        {index: (h, w, 4) float32}."""
        d = np.ascontiguousarray(d_image, np.float32)
        n = len(self.scene.images)
        images = range(n) if images is None else images
        outs = {k: np.zeros(self.scene.images[k].shape[:2] + (4,), np.float32) for k in images}
        ptrs = (C.c_void_p * max(n, 1))(*[outs[k].ctypes.data if k in outs else None for k in range(n)])
        st = _abi.S2RenderStats()
        self._check(self._lib.s2_render_adjoint(self._h, C.byref(view), C.byref(params), d.ctypes.data, 1,
                                                C.cast(ptrs, C.c_void_p), C.byref(st)))
        return outs

    def render_adjoint_device(self, view, params: _abi.S2RenderParams, d_ptr: int, grad_ptrs) -> _abi.S2RenderStats:
        """Device variant: grad_ptrs is one device pointer (or None) per scene image."""
        ptrs = (C.c_void_p * max(len(grad_ptrs), 1))(*grad_ptrs)
        st = _abi.S2RenderStats()
        self._check(self._lib.s2_render_adjoint(self._h, C.byref(view), C.byref(params), C.c_void_p(d_ptr), 0,
                                                C.cast(ptrs, C.c_void_p), C.byref(st)))
        return st

    def cache_query_device(self, pos_ptr: int, n: int, out_ptr: int):
        """Cache inference on device buffers (float4 positions in, float4 radiance out)."""
        self._check(self._lib.s2_cache_query(self._h, C.c_void_p(pos_ptr), n, C.c_void_p(out_ptr), 1))

    def cache_train_device(self, pos_ptr: int, target_ptr: int, n: int) -> float:
        """One optimiser step on device records (float4 positions, float4 targets); mean loss."""
        loss = C.c_float(0)
        self._check(self._lib.s2_cache_train(self._h, C.c_void_p(pos_ptr), C.c_void_p(target_ptr), n, C.byref(loss), 1))
        return loss.value

    # ---- tuning
    # ---- post-processing (device buffers, e.g. torch tensors' data_ptr())
    @staticmethod
    def default_temporal_params() -> _abi.S2TemporalParams:
        p = _abi.S2TemporalParams()
        _abi.lib().s2_default_temporal_params(C.byref(p))
        return p

    def temporal_accumulate(self, view, params: _abi.S2TemporalParams, frame: _abi.S2Aovs, accum_color_ptr: int,
                            accum_moments_ptr: int | None = None, instance_index_map_ptr: int | None = None):
        """One frame of temporal accumulation (s2_temporal_accumulate) over the device AOVs in `frame`."""
        self._check(self._lib.s2_temporal_accumulate(self._h, C.byref(view), C.byref(params), C.byref(frame),
                                                     C.c_void_p(instance_index_map_ptr) if instance_index_map_ptr else None,
                                                     C.c_void_p(accum_color_ptr),
                                                     C.c_void_p(accum_moments_ptr) if accum_moments_ptr else None))

    @staticmethod
    def default_svgf_params() -> _abi.S2SvgfParams:
        p = _abi.S2SvgfParams()
        _abi.lib().s2_default_svgf_params(C.byref(p))
        return p

    def svgf_filter(self, view, params: _abi.S2SvgfParams, frame: _abi.S2Aovs, output_ptr: int,
                    instance_index_map_ptr: int | None = None):
        """SVGF variance estimate + a-trous passes over the accumulation history (s2_svgf_filter)."""
        self._check(self._lib.s2_svgf_filter(self._h, C.byref(view), C.byref(params), C.byref(frame),
                                             C.c_void_p(instance_index_map_ptr) if instance_index_map_ptr else None,
                                             C.c_void_p(output_ptr)))

    def tonemap(self, width: int, height: int, params: _abi.S2TonemapParams, input_ptr: int, output_ptr: int,
                albedo_ptr: int | None = None):
        """Tonemaps a device float4 image (s2_tonemap)."""
        self._check(self._lib.s2_tonemap(self._h, width, height, C.byref(params), C.c_void_p(input_ptr),
                                         C.c_void_p(albedo_ptr) if albedo_ptr else None, C.c_void_p(output_ptr)))

    def set_tuning(self, tuning: _abi.S2Tuning | None):
        self._check(self._lib.s2_set_tuning(self._h, C.byref(tuning) if tuning is not None else None))

    def get_tuning(self) -> _abi.S2Tuning:
        t = _abi.S2Tuning()
        self._check(self._lib.s2_get_tuning(self._h, C.byref(t)))
        return t

    def autotune(self, view, params: _abi.S2RenderParams) -> tuple[_abi.S2Tuning, int]:
        """Measures tuning candidates on this scene/view/params and applies the fastest."""
        t = _abi.S2Tuning()
        n = C.c_uint32(0)
        self._check(self._lib.s2_autotune(self._h, C.byref(view), C.byref(params), C.byref(t), C.byref(n)))
        return t, n.value
