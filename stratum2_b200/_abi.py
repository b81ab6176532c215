"""ctypes mirror of include/stratum2.h.

Loading fails loudly when the CUDA library is missing: there is no CPU fallback for the product
path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "libstratum2_b200.so"

ABI_VERSION = 2  # S2_ABI_VERSION

S2_OK = 0
S2_ERR_INVALID = -1
S2_ERR_CUDA = -2
S2_ERR_OOM = -3
S2_ERR_NO_SCENE = -4
S2_ERR_TIMEOUT = -5
S2_ERR_DEVICE = -6
S2_ERR_UNSUPPORTED = -7

INVALID_INDEX16 = 0xFFFF
INVALID_INDEX32 = 0xFFFFFFFF
NO_BUFFER = 0xFFFF
NO_IMAGE = 0xFFFFFFFF
NO_ENVIRONMENT = 0xFFFFFFFF

FLAG_PIXEL_JITTER = 1 << 0
FLAG_LAMBERTIAN = 1 << 1
FLAG_PCG32 = 1 << 2
FLAG_NO_NEE = 1 << 3
FLAG_RESTIR_DI = 1 << 4
FLAG_REFERENCE_ENV_MIS = 1 << 5
FLAG_NO_RR = 1 << 6
FLAG_ACCUMULATE = 1 << 7
FLAG_SHADING_NORMALS_OFF = 1 << 8
FLAG_PROFILE_KERNELS = 1 << 9
FLAG_COUNT_FETCHES = 1 << 10
FLAG_RESTIR_REUSE = 1 << 11
FLAG_ALPHA_TEST_OFF = 1 << 12
FLAG_NORMAL_MAPS_OFF = 1 << 13
FLAG_RADIANCE_CACHE = 1 << 14
FLAG_RESTIR_SCREEN = 1 << 15
FLAG_LIGHT_POWER_PICK = 1 << 16
FLAG_LIGHT_TRACE = 1 << 17
FLAG_ENV_FOOTPRINT_PDF = 1 << 19
FLAG_RESTIR_REUSE_VISIBILITY = 1 << 18
SHADE_ORDER_MATERIAL = 0
SHADE_ORDER_QUEUE = 1
TRACE_ORDER_QUEUE = 0
TRACE_ORDER_COHERENT = 1
SHADE_RECORDS_ON = 0
SHADE_RECORDS_OFF = 1
SHADOW_MERGE_ON = 0
SHADOW_MERGE_OFF = 1
BVH_COLLAPSE_SAH = 0
BVH_COLLAPSE_GREEDY = 1

# every symbol include/stratum2.h declares
EXPORTED_SYMBOLS = [
    "s2_get_abi_version", "s2_create", "s2_destroy", "s2_last_error", "s2_sync", "s2_set_stream",
    "s2_scene_upload", "s2_build_bvh", "s2_get_bvh", "s2_trace", "s2_trace_counted", "s2_render",
    "s2_default_render_params", "s2_render_noalloc", "s2_render_views",
    "s2_cache_default_params", "s2_cache_init", "s2_cache_get_params", "s2_cache_set_params", "s2_cache_query",
    "s2_cache_train", "s2_cache_gradients", "s2_update_image", "s2_render_diff", "s2_render_adjoint",
    "s2_set_tuning", "s2_get_tuning", "s2_autotune",
    "s2_default_temporal_params", "s2_temporal_accumulate", "s2_tonemap", "s2_default_svgf_params", "s2_svgf_filter",
    "s2_default_vcm_params", "s2_render_vcm", "s2_device_math", "s2_inject_wait_timeout",
    "s2_repack_metallic_roughness",
]

CACHE_WEIGHTS = 6336
CACHE_LEVELS = 16


class S2Image(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("channels", C.c_uint32),
                ("texels", C.POINTER(C.c_float))]


class S2SceneDesc(C.Structure):
    _fields_ = [
        ("instance_count", C.c_uint32),
        ("instances", C.POINTER(C.c_uint32)),
        ("primitive_counts", C.POINTER(C.c_uint32)),
        ("transforms", C.POINTER(C.c_float)),
        ("inverse_transforms", C.POINTER(C.c_float)),
        ("motion_transforms", C.POINTER(C.c_float)),
        ("vertex_info_count", C.c_uint32),
        ("vertex_infos", C.POINTER(C.c_uint32)),
        ("vertex_buffer_count", C.c_uint32),
        ("vertex_buffers", C.POINTER(C.c_void_p)),
        ("vertex_buffer_bytes", C.POINTER(C.c_uint64)),
        ("material_bytes", C.c_uint32),
        ("material_data", C.c_void_p),
        ("light_count", C.c_uint32),
        ("light_instance_map", C.POINTER(C.c_uint32)),
        ("instance_light_map", C.POINTER(C.c_uint32)),
        ("environment_material_address", C.c_uint32),
        ("image_count", C.c_uint32),
        ("images", C.POINTER(S2Image)),
        ("scene_sphere", C.c_float * 4),
    ]


class S2BvhParams(C.Structure):
    _fields_ = [("max_leaf_size", C.c_uint32), ("sah_bins", C.c_uint32), ("threads", C.c_uint32),
                ("collapse", C.c_uint32)]


class S2BvhStats(C.Structure):
    _fields_ = [("node_count", C.c_uint64), ("triangle_count", C.c_uint64), ("leaf_slot_count", C.c_uint64),
                ("max_depth", C.c_uint32), ("reserved", C.c_uint32), ("build_seconds", C.c_double),
                ("sah_cost", C.c_double)]


class S2Ray(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("tmin", C.c_float), ("direction", C.c_float * 3), ("tmax", C.c_float)]


class S2Hit(C.Structure):
    _fields_ = [("t", C.c_float), ("instance", C.c_uint32), ("primitive", C.c_uint32),
                ("barycentrics", C.c_float * 2)]


class S2View(C.Structure):
    _fields_ = [("projection", C.c_float * 8), ("image_min", C.c_int32 * 2), ("image_max", C.c_int32 * 2),
                ("camera_to_world", C.c_float * 12), ("prev_world_to_camera", C.c_float * 12)]


class S2RenderParams(C.Structure):
    _fields_ = [
        ("min_path_length", C.c_uint32), ("max_path_length", C.c_uint32), ("exposure", C.c_float),
        ("spp", C.c_uint32), ("frame_seed", C.c_uint32), ("flags", C.c_uint32),
        ("environment_sample_probability", C.c_float), ("restir_candidates", C.c_uint32),
        ("restir_max_m", C.c_float), ("wave_paths", C.c_uint32), ("restir_grid_cells", C.c_uint32),
        ("restir_grid_cell_size", C.c_float), ("restir_grid_pixel_radius", C.c_float),
        ("cache_bounces", C.c_uint32), ("cache_train_paths", C.c_uint32), ("restir_spatial", C.c_uint32),
        ("restir_spatial_radius", C.c_float), ("light_subpaths", C.c_float),
        ("cache_min_roughness", C.c_float), ("reserved", C.c_uint32),
    ]


class S2Aovs(C.Structure):
    _fields_ = [("radiance", C.c_void_p), ("albedo", C.c_void_p), ("visibility", C.c_void_p),
                ("depth", C.c_void_p), ("prev_uv", C.c_void_p), ("ids32", C.c_void_p)]


class S2CacheParams(C.Structure):
    _fields_ = [("box_min", C.c_float * 3), ("box_max", C.c_float * 3), ("log2_table", C.c_uint32),
                ("base_resolution", C.c_uint32), ("max_resolution", C.c_uint32), ("learning_rate", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("epsilon", C.c_float), ("seed", C.c_uint32),
                ("reserved", C.c_uint32 * 6)]


class S2Tuning(C.Structure):
    _fields_ = [("wave_paths", C.c_uint32), ("trav_tris_per_step", C.c_uint32), ("trav_vote8", C.c_uint32),
                ("refill_min", C.c_uint32), ("shade_order", C.c_uint32), ("trace_order", C.c_uint32),
                ("shade_records", C.c_uint32), ("shadow_merge", C.c_uint32)]


TEMPORAL_REPROJECT, TEMPORAL_CHECK_NORMAL, TEMPORAL_CHECK_DEPTH = 1 << 0, 1 << 1, 1 << 2
TEMPORAL_DEMODULATE_ALBEDO, TEMPORAL_SHADOW_HYSTERESIS, TEMPORAL_RESET = 1 << 3, 1 << 4, 1 << 5
(TONEMAP_RAW, TONEMAP_REINHARD, TONEMAP_REINHARD_EXTENDED, TONEMAP_REINHARD_LUMINANCE, TONEMAP_REINHARD_LUMINANCE_EXT,
 TONEMAP_UNCHARTED2, TONEMAP_FILMIC, TONEMAP_ACES, TONEMAP_ACES_APPROX, TONEMAP_VIRIDIS_R,
 TONEMAP_VIRIDIS_LENGTH_RGB) = range(11)
TONEMAP_GAMMA, TONEMAP_GAMMA_REFERENCE = 1 << 0, 1 << 1


class S2TemporalParams(C.Structure):
    _fields_ = [("flags", C.c_uint32), ("history_limit", C.c_uint32), ("shadow_preserve_offset", C.c_float),
                ("shadow_preserve_scale", C.c_float)]


(SVGF_KERNEL_ATROUS, SVGF_KERNEL_BOX3, SVGF_KERNEL_BOX5, SVGF_KERNEL_SUBSAMPLED, SVGF_KERNEL_BOX3_SUBSAMPLED,
 SVGF_KERNEL_BOX5_SUBSAMPLED) = range(6)


class S2SvgfParams(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("kernel", C.c_uint32), ("history_tap", C.c_uint32), ("flags", C.c_uint32),
                ("history_limit", C.c_uint32), ("variance_boost_length", C.c_float), ("sigma_luminance_boost", C.c_float),
                ("reserved", C.c_uint32)]


class S2TonemapParams(C.Structure):
    _fields_ = [("mode", C.c_uint32), ("exposure", C.c_float), ("flags", C.c_uint32), ("reserved", C.c_uint32)]


# vertex connection and merging (S2_VCM_*)
VCM_PATH_TRACE, VCM_LIGHT_TRACE, VCM_PPM, VCM_BPM, VCM_BPT, VCM_VCM = range(6)
VCM_FLAG_LIGHT_VERTEX_CACHE, VCM_FLAG_DEBUG_PATHS, VCM_FLAG_DEBUG_UNWEIGHTED = 1 << 0, 1 << 1, 1 << 2
VCM_FLAG_DI_RIS, VCM_FLAG_DI_REUSE, VCM_FLAG_LVC_RIS, VCM_FLAG_LVC_REUSE = 1 << 3, 1 << 4, 1 << 5, 1 << 6


class S2VcmParams(C.Structure):
    _fields_ = [("algorithm", C.c_uint32), ("min_path_length", C.c_uint32), ("max_path_length", C.c_uint32),
                ("iterations", C.c_uint32), ("frame_seed", C.c_uint32), ("first_iteration", C.c_uint32),
                ("flags", C.c_uint32), ("vcm_flags", C.c_uint32), ("light_path_fraction", C.c_float),
                ("merge_radius_factor", C.c_float), ("merge_radius_alpha", C.c_float), ("exposure", C.c_float),
                ("debug_camera_vertices", C.c_uint16), ("debug_light_vertices", C.c_uint16),
                ("di_candidates", C.c_uint32), ("di_max_m", C.c_float), ("lvc_candidates", C.c_uint32),
                ("lvc_max_m", C.c_float)]


class S2RenderStats(C.Structure):
    _fields_ = [("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("paths", C.c_uint64),
                ("nan_count", C.c_uint64), ("gpu_ms", C.c_double), ("kernel_launches", C.c_uint64),
                ("extend_ms", C.c_double), ("shade_ms", C.c_double), ("occlude_ms", C.c_double),
                ("extend_launches", C.c_uint32), ("shade_launches", C.c_uint32), ("occlude_launches", C.c_uint32),
                ("reserved", C.c_uint32), ("extend_node_fetches", C.c_uint64), ("extend_tri_fetches", C.c_uint64),
                ("shadow_node_fetches", C.c_uint64), ("shadow_tri_fetches", C.c_uint64)]


assert C.sizeof(S2Ray) == 32 and C.sizeof(S2Hit) == 20
assert C.sizeof(S2RenderParams) == 80
assert C.sizeof(S2CacheParams) == 80
assert C.sizeof(S2VcmParams) == 68

_lib = None


def lib() -> C.CDLL:
    """Loads libstratum2_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise RuntimeError(f"{_LIB_PATH} is missing: build it with `python -m stratum2_b200.build`")
    L = C.CDLL(str(_LIB_PATH))
    P = C.POINTER
    L.s2_get_abi_version.restype = C.c_int
    L.s2_create.argtypes = [C.c_int, P(C.c_void_p)]
    L.s2_destroy.argtypes = [C.c_void_p]
    L.s2_destroy.restype = None
    L.s2_device_math.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_uint32, C.c_void_p]
    L.s2_inject_wait_timeout.argtypes = [C.c_void_p, C.c_uint32]
    L.s2_last_error.argtypes = [C.c_void_p]
    L.s2_last_error.restype = C.c_char_p
    L.s2_sync.argtypes = [C.c_void_p]
    L.s2_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    L.s2_scene_upload.argtypes = [C.c_void_p, P(S2SceneDesc)]
    L.s2_build_bvh.argtypes = [C.c_void_p, P(S2BvhParams), P(S2BvhStats)]
    L.s2_trace.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p, C.c_int]
    L.s2_trace_counted.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
    L.s2_get_bvh.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.s2_render.argtypes = [C.c_void_p, P(S2View), P(S2RenderParams), P(S2Aovs), C.c_int, P(S2RenderStats)]
    L.s2_render_views.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, P(S2RenderParams), C.c_void_p, C.c_int,
                                  P(S2RenderStats)]
    L.s2_render_noalloc.argtypes = [C.c_void_p, P(S2View), P(S2RenderParams), P(S2Aovs), P(S2RenderStats)]
    L.s2_default_render_params.argtypes = [P(S2RenderParams)]
    L.s2_default_render_params.restype = None
    L.s2_update_image.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_int]
    L.s2_repack_metallic_roughness.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32), C.c_int]
    L.s2_set_tuning.argtypes = [C.c_void_p, P(S2Tuning)]
    L.s2_default_temporal_params.restype = None
    L.s2_default_temporal_params.argtypes = [P(S2TemporalParams)]
    L.s2_temporal_accumulate.argtypes = [C.c_void_p, P(S2View), P(S2TemporalParams), P(S2Aovs), C.c_void_p, C.c_void_p,
                                         C.c_void_p]
    L.s2_default_svgf_params.restype = None
    L.s2_default_svgf_params.argtypes = [P(S2SvgfParams)]
    L.s2_svgf_filter.argtypes = [C.c_void_p, P(S2View), P(S2SvgfParams), P(S2Aovs), C.c_void_p, C.c_void_p]
    L.s2_tonemap.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, P(S2TonemapParams), C.c_void_p, C.c_void_p, C.c_void_p]
    L.s2_get_tuning.argtypes = [C.c_void_p, P(S2Tuning)]
    L.s2_autotune.argtypes = [C.c_void_p, P(S2View), P(S2RenderParams), P(S2Tuning), P(C.c_uint32)]
    L.s2_default_vcm_params.restype = None
    L.s2_default_vcm_params.argtypes = [P(S2VcmParams)]
    L.s2_render_vcm.argtypes = [C.c_void_p, P(S2View), P(S2VcmParams), P(S2Aovs), C.c_int, P(S2RenderStats)]
    L.s2_render_diff.argtypes = [C.c_void_p, P(S2View), P(S2RenderParams), C.c_void_p, C.c_int, P(S2RenderStats)]
    L.s2_render_adjoint.argtypes = [C.c_void_p, P(S2View), P(S2RenderParams), C.c_void_p, C.c_int, C.c_void_p,
                                    P(S2RenderStats)]
    L.s2_cache_default_params.argtypes = [P(S2CacheParams)]
    L.s2_cache_default_params.restype = None
    L.s2_cache_init.argtypes = [C.c_void_p, P(S2CacheParams)]
    L.s2_cache_get_params.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.s2_cache_set_params.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.s2_cache_query.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_int]
    L.s2_cache_train.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, P(C.c_float), C.c_int]
    L.s2_cache_gradients.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                     P(C.c_float), C.c_int]
    for name in EXPORTED_SYMBOLS:
        getattr(L, name)
    if L.s2_get_abi_version() != ABI_VERSION:
        raise RuntimeError(f"{_LIB_PATH} has ABI {L.s2_get_abi_version()}, expected {ABI_VERSION}: rebuild it")
    _lib = L
    return L


class S2Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"stratum2 error {code}: {msg}")
        self.code = code
