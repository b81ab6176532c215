/*
 * stratum2.h -- C ABI of the B200 path-tracing hot path (unidirectional path tracing with
 * next-event estimation and ReSTIR DI), a drop-in for the renderer path of Shmaug/Stratum2.
 *
 * Every entry point returns an int status (S2_OK == 0, negative S2_ERR_* on failure), never
 * throws and never aborts.  s2_last_error() returns a message for the last failing call on a
 * context.  All structs are plain C: pointers, sizes and fixed-width integers; no C++ or torch
 * types cross this boundary.
 *
 * Reference interfaces replaced (paths relative to the Stratum2 source tree):
 *   - scene buffers:  Scene::FrameData descriptors bound to SceneParameters
 *                     (src/App/Scene.cpp:768-790, src/Shaders/common/scene.hlsli:6-41)
 *   - renderer:       TestRenderer::render(CommandBuffer&, const Image::View&)
 *                     (src/App/TestRenderer.hpp:20, src/App/TestRenderer.cpp:284-763)
 *                     VCM::render in kPathTrace mode for minPathLength/maxPathLength
 *                     (src/App/VCM.cpp:39-40)
 *   - ray queries:    traceRay / traceVisibilityRay (src/Shaders/common/intersection.hlsli:68-338)
 *   - exposure:       Tonemapper --exposure (src/App/Tonemapper.cpp:25, kernels/tonemap.slang:154)
 */
#ifndef STRATUM2_H_
#define STRATUM2_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define S2_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------------------------ */
#define S2_OK               0
#define S2_ERR_INVALID     -1  /* bad argument (null pointer, size, unknown flag) */
#define S2_ERR_CUDA        -2  /* a CUDA runtime call failed */
#define S2_ERR_OOM         -3  /* device allocation failed or allocation budget exceeded */
#define S2_ERR_NO_SCENE    -4  /* render/trace before s2_scene_upload + s2_build_bvh */
#define S2_ERR_TIMEOUT     -5  /* a bounded device wait gave up (status word set by a kernel) */
#define S2_ERR_DEVICE      -6  /* a kernel reported an internal error (stack/queue overflow) */
#define S2_ERR_UNSUPPORTED -7  /* feature not supported on this device / build */

/* ---- reference-format constants (src/Shaders/compat/scene.h:13-24) ---------------------- */
#define S2_INVALID_INDEX16       0xFFFFu      /* INVALID_INSTANCE / INVALID_PRIMITIVE */
#define S2_INVALID_INDEX32       0xFFFFFFFFu
#define S2_INSTANCE_TYPE_MESH    0u
#define S2_INSTANCE_TYPE_SPHERE  1u           /* accepted, not rendered (no spheres on this path) */
#define S2_INSTANCE_TYPE_VOLUME  2u           /* accepted, not rendered (no media on this path) */
#define S2_NO_BUFFER             0xFFFFu      /* MeshVertexInfo buffer index meaning "absent" */
#define S2_NO_IMAGE              0xFFFFFFFFu  /* material / environment image index "absent" */
#define S2_NO_ENVIRONMENT        0xFFFFFFFFu  /* environment material address "absent" */
#define S2_MATERIAL_RECORD_BYTES 64u          /* Material::store (src/App/Material.hpp:22-38) */

typedef struct S2Context S2Context;

/* A float image: RGBA (channels 4), RG (2) or R (1) texels, row-major, level 0 only. Mip levels
 * needed by environment importance sampling are built on the device by 2x2 averaging. */
typedef struct S2Image {
    uint32_t width, height, channels;
    const float* texels;           /* host pointer, width*height*channels floats */
} S2Image;

/* Packed scene, byte-compatible with the reference's frame data:
 *   instances          InstanceData[n] = {type:4 | materialAddress:28, data}   (compat/scene.h:30-58)
 *                      mesh data = vertexInfoIndex:16 | primitiveCount:16
 *   primitive_counts   optional u32[n]: 32-bit primitive counts that override the 16-bit field,
 *                      so one instance may hold more than 65,535 triangles
 *   transforms         TransformData[n] = row-major float 3x4 object-to-world (compat/transform.h:7)
 *   inverse/motion     optional (NULL => computed / identity motion)
 *   vertex_infos       MeshVertexInfo[] = 8 x u32 each (compat/scene.h:89-132)
 *   vertex_buffers     ByteAddressBuffer[]: indices (u16/u32), float3 positions/normals, float2 uvs
 *   material_data      byte-address buffer of 64-B material records plus the 16-B environment
 *                      record {float3 emission scale, u32 image} (src/App/Scene.hpp:41-45)
 *   light maps         mLightInstanceMap / mInstanceLightMap (src/App/Scene.cpp:441-491)
 */
typedef struct S2SceneDesc {
    uint32_t instance_count;
    const uint32_t* instances;            /* 2*instance_count */
    const uint32_t* primitive_counts;     /* optional, instance_count */
    const float* transforms;              /* 12*instance_count */
    const float* inverse_transforms;      /* optional, 12*instance_count */
    const float* motion_transforms;       /* optional, 12*instance_count */

    uint32_t vertex_info_count;
    const uint32_t* vertex_infos;         /* 8*vertex_info_count */

    uint32_t vertex_buffer_count;
    const void* const* vertex_buffers;    /* host pointers */
    const uint64_t* vertex_buffer_bytes;

    uint32_t material_bytes;
    const void* material_data;

    uint32_t light_count;
    const uint32_t* light_instance_map;   /* light_count */
    const uint32_t* instance_light_map;   /* optional, instance_count */

    uint32_t environment_material_address; /* S2_NO_ENVIRONMENT if none */

    uint32_t image_count;
    const S2Image* images;

    float scene_sphere[4];                /* center xyz, radius (TestRenderer.cpp:458-461) */
} S2SceneDesc;

/* BVH8 build parameters (the reference delegates this to vkCmdBuildAccelerationStructuresKHR,
 * src/App/Scene.cpp:17-55). */
typedef struct S2BvhParams {
    uint32_t max_leaf_size;   /* triangles per BVH8 leaf slot, 1..3 (default 3) */
    uint32_t sah_bins;        /* binned-SAH bins (default 32) */
    uint32_t threads;         /* host build threads (0 = all) */
    uint32_t collapse;        /* S2_BVH_COLLAPSE_SAH (0, default): the binary tree is collapsed into
                                 8-wide nodes by a cost-optimal dynamic program over the surface-area
                                 cost; S2_BVH_COLLAPSE_GREEDY (1): by repeatedly opening the child of
                                 largest area */
} S2BvhParams;
#define S2_BVH_COLLAPSE_SAH    0u
#define S2_BVH_COLLAPSE_GREEDY 1u

typedef struct S2BvhStats {
    uint64_t node_count, triangle_count, leaf_slot_count;
    uint32_t max_depth, reserved;
    double build_seconds;
    double sah_cost;
} S2BvhStats;

/* Ray and hit for the parity / query entry point s2_trace. */
typedef struct S2Ray {
    float origin[3];
    float tmin;
    float direction[3];
    float tmax;
} S2Ray;                                   /* 32 B */

typedef struct S2Hit {
    float t;                               /* distance, or tmax when missed */
    uint32_t instance;                     /* S2_INVALID_INDEX32 when missed */
    uint32_t primitive;
    float barycentrics[2];                 /* weights of vertex 1 and vertex 2 */
} S2Hit;                                   /* 20 B */

/* A pinhole view: ViewData + camera TransformData (compat/scene.h:134-167, transform.h:128-190).
 * The camera looks down -z of its transform; projection is the reference's reversed-z
 * perspective (makePerspective, transform.h:181-190). */
typedef struct S2View {
    float projection[8];      /* ProjectionData: scale.xy, offset.xy, near, far, sensorArea, vfov */
    int32_t image_min[2];
    int32_t image_max[2];
    float camera_to_world[12];
    float prev_world_to_camera[12];  /* previous frame's inverse transform (prev-UV AOV) */
} S2View;

/* Render flags */
#define S2_FLAG_PIXEL_JITTER        (1u << 0)  /* gPixelJitter (off in the reference) */
#define S2_FLAG_LAMBERTIAN          (1u << 1)  /* gLambertian: Lambertian instead of Disney */
#define S2_FLAG_PCG32               (1u << 2)  /* PCG32 per-pixel stream instead of pcg4d */
#define S2_FLAG_NO_NEE              (1u << 3)  /* disable gSampleDirectIllumination */
#define S2_FLAG_RESTIR_DI           (1u << 4)  /* gReSTIR_DI: RIS over candidate light samples */
#define S2_FLAG_REFERENCE_ENV_MIS   (1u << 5)  /* BSDF-hit environment MIS with the disc pdf 1/(pi R^2)
                                                  as the reference does (testrenderer.slang:1047-1050) */
#define S2_FLAG_NO_RR               (1u << 6)  /* disable Russian roulette */
#define S2_FLAG_ACCUMULATE          (1u << 7)  /* add into the previous accumulation (progressive) */
#define S2_FLAG_SHADING_NORMALS_OFF (1u << 8)  /* ignore vertex normals (gShadingNormals false) */
#define S2_FLAG_PROFILE_KERNELS     (1u << 9)  /* time extend/shade/occlude launches with CUDA events */
#define S2_FLAG_COUNT_FETCHES       (1u << 10) /* count BVH node and triangle fetches (slower) */
#define S2_FLAG_RESTIR_REUSE        (1u << 11) /* gReSTIR_DI_Reuse: with S2_FLAG_RESTIR_DI, reuse one
                                                  reservoir per vertex from the previous s2_render
                                                  call's world-space hash grid and store this call's
                                                  reservoirs for the next call (testrenderer.slang:
                                                  608-726).  Results depend on atomic append order. */
#define S2_FLAG_ALPHA_TEST_OFF      (1u << 12) /* disable gAlphaTest (on in the reference) */
#define S2_FLAG_NORMAL_MAPS_OFF     (1u << 13) /* disable gNormalMaps (on in the reference) */
#define S2_FLAG_RADIANCE_CACHE      (1u << 14) /* learned radiance cache (no counterpart in the
                                                  reference; needs s2_cache_init): paths end at
                                                  vertex cache_bounces + 1 with the cache's
                                                  scattered radiance there, and one path in
                                                  (paths / cache_train_paths) runs to its end and
                                                  trains the cache after each wave; in
                                                  s2_render_views the cache_train_paths training
                                                  paths are extra paths with their own
                                                  accumulators, and training follows each call */
#define S2_FLAG_RESTIR_SCREEN       (1u << 15) /* screen-space ReSTIR DI reuse (no counterpart in the
                                                  reference, which reuses through the hash grid of
                                                  S2_FLAG_RESTIR_REUSE; exclusive with it): with
                                                  S2_FLAG_RESTIR_DI, the primary vertex of every path
                                                  combines its RIS reservoir with the previous
                                                  s2_render call's reservoirs at its reprojected
                                                  pixel (temporal) and at restir_spatial random pixels
                                                  within restir_spatial_radius of it (spatial); each
                                                  pixel's sample-0 path stores its reservoir for the
                                                  next call (s2_render only) */
#define S2_FLAG_RESTIR_REUSE_VISIBILITY (1u << 18) /* gReSTIR_DI_Reuse_Visibility (TestRenderer.cpp:34,
                                                   testrenderer.slang:611-742): with reuse on, the
                                                   canonical sample's visibility is traced before
                                                   reuse (occluded: W = 0), a reused sample's in the
                                                   current domain before resampling, and the result
                                                   is added without a deferred shadow ray; ignored
                                                   without S2_FLAG_RESTIR_REUSE / _SCREEN */
#define S2_FLAG_LIGHT_TRACE         (1u << 17) /* TestRenderer's light tracing mode (mLightTrace,
                                                  testrenderer.slang:441-512, 983-1020): light
                                                  subpaths connect every non-singular vertex to the
                                                  camera; no NEE, ReSTIR or cache; the radiance AOV
                                                  is written, the others are cleared to zero
                                                  (s2_render only) */
#define S2_FLAG_ENV_FOOTPRINT_PDF   (1u << 19) /* importance-sample the environment by the largest
                                                  luminance its bilinear reconstruction takes over each
                                                  texel (tables built at s2_scene_upload) instead of
                                                  the texel's own luminance, as the reference does
                                                  (lights.hlsli:49-138); no counterpart in the
                                                  reference.  Same expected image: the environment is
                                                  evaluated bilinearly, so near a small bright source
                                                  (a sun of one texel) the texel pdf leaves its
                                                  interpolated halo to BSDF sampling, whose rare hits
                                                  are fireflies; this pdf covers the halo */
#define S2_FLAG_LIGHT_POWER_PICK    (1u << 16) /* pick emissive lights in proportion to their power
                                                  (emission luminance x area, from an alias table built
                                                  at s2_scene_upload) instead of uniformly as the
                                                  reference does (lights.hlsli:200); no counterpart in
                                                  the reference.  Same expected image, less noise with
                                                  many lights of unequal power */

typedef struct S2RenderParams {
    uint32_t min_path_length;        /* VCM --minPathLength (vcm.slang:922,960,977) */
    uint32_t max_path_length;        /* mMaxDepth / --maxPathLength */
    float exposure;                  /* radiance *= 2^exposure on output */
    uint32_t spp;                    /* samples per pixel in this call */
    uint32_t frame_seed;             /* sample s uses RNG seed frame_seed + s (mRandomSeed) */
    uint32_t flags;                  /* S2_FLAG_* */
    float environment_sample_probability; /* default 0.9 (TestRenderer.cpp:41) */
    uint32_t restir_candidates;      /* mCandidateSamples (default 32) */
    float restir_max_m;              /* mMaxM (default 3) */
    uint32_t wave_paths;             /* paths in flight per wave / queue (0 = 2^26) */
    uint32_t restir_grid_cells;      /* hash-grid cell count (0 = 100000, TestRenderer.cpp:52) */
    float restir_grid_cell_size;     /* minimum cell size (0 = 0.5, TestRenderer.cpp:52) */
    float restir_grid_pixel_radius;  /* mCellPixelRadius: 0 = constant cell size */
    uint32_t cache_bounces;          /* S2_FLAG_RADIANCE_CACHE: bounces before the cache (0 = 2) */
    uint32_t cache_train_paths;      /* training paths per wave (0 = 65536) */
    uint32_t restir_spatial;         /* S2_FLAG_RESTIR_SCREEN: spatial neighbours (0 = 5, at most 32) */
    float restir_spatial_radius;     /* S2_FLAG_RESTIR_SCREEN: neighbour radius in pixels (0 = 30) */
    float light_subpaths;            /* S2_FLAG_LIGHT_TRACE: light subpaths per sample pass =
                                        max(1, pixels x light_subpaths) (mLightSubpathCount, 0 = 1) */
    float cache_min_roughness;       /* S2_FLAG_RADIANCE_CACHE: path regularisation (no counterpart in
                                        the reference).  The roughness of every path vertex after the
                                        first is raised to at least this value, so reflections of small
                                        bright lights reached through a bounce (caustics, double glossy
                                        reflections of the sun) are blurred instead of sampled as rare
                                        fireflies; the first vertex is untouched.  Biased, as the cache
                                        itself is; 0 = off (default) */
    uint32_t reserved;
} S2RenderParams;

/* Output AOVs (caller-allocated, device or host pointers per s2_render's `out_on_host`).
 * Any pointer may be NULL to skip that AOV.  Layouts follow TestRenderer's images
 * (TestRenderer.cpp:323-347, testrenderer.slang:195-218). */
typedef struct S2Aovs {
    float* radiance;        /* float4 per pixel: mean radiance * 2^exposure, w = 1 */
    float* albedo;          /* float4 per pixel: baseColor at the first hit, 1 on a miss */
    uint32_t* visibility;   /* uint2 per pixel: {instance:16 | primitive:16, packed shading normal} */
    float* depth;           /* float4 per pixel: {depth, prevDepth, 1, 1} */
    float* prev_uv;         /* float2 per pixel */
    uint32_t* ids32;        /* uint2 per pixel: {instance, primitive} as 32-bit ids */
} S2Aovs;

/* Per-call statistics (device counters, read back after the call). */
typedef struct S2RenderStats {
    uint64_t extension_rays;   /* closest-hit rays traced */
    uint64_t shadow_rays;      /* any-hit rays traced */
    uint64_t paths;            /* camera paths (pixels x spp) */
    uint64_t nan_count;        /* paths dropped for NaN/Inf throughput */
    double gpu_ms;             /* device time of the call (CUDA events) */
    uint64_t kernel_launches;  /* kernels launched by the call */
    /* S2_FLAG_PROFILE_KERNELS: summed device time per kernel kind */
    double extend_ms, shade_ms, occlude_ms;
    uint32_t extend_launches, shade_launches, occlude_launches, reserved;
    /* S2_FLAG_COUNT_FETCHES: BVH node / triangle fetches of extension and shadow rays */
    uint64_t extend_node_fetches, extend_tri_fetches, shadow_node_fetches, shadow_tri_fetches;
} S2RenderStats;

/* ---- lifecycle --------------------------------------------------------------------------- */
int  s2_get_abi_version(void);
int  s2_create(int device, S2Context** out);
void s2_destroy(S2Context* ctx);
const char* s2_last_error(const S2Context* ctx);
int  s2_sync(S2Context* ctx);
/* Use `stream` (a cudaStream_t) for all work of this context; NULL = the context's own stream. */
int  s2_set_stream(S2Context* ctx, void* stream);

/* ---- scene ------------------------------------------------------------------------------- */
/* Copies the packed scene to the device (inputs are host pointers; the caller keeps ownership). */
int  s2_scene_upload(S2Context* ctx, const S2SceneDesc* scene);
/* Builds the BVH8 over all mesh instances (flattened to world space). */
int  s2_build_bvh(S2Context* ctx, const S2BvhParams* params, S2BvhStats* stats_out);
/* Copies the built BVH8 to host memory: `nodes` receives counts_out[0] 128-byte nodes and `tris`
 * counts_out[1] 48-byte triangle records (layouts: stratum2_b200/csrc/s2_bvh.h).  Either pointer
 * may be NULL (call once with both NULL to size the buffers). */
int  s2_get_bvh(S2Context* ctx, void* nodes, void* tris, uint64_t* counts_out);

/* ---- queries (replace traceRay / traceVisibilityRay) ------------------------------------- */
/* rays/hits are DEVICE pointers when on_device != 0, else host pointers.
 * anyhit != 0: first-hit query (RAY_FLAG_ACCEPT_FIRST_HIT_AND_END_SEARCH); hit.t is then the
 * found hit's distance and only hit.instance != S2_INVALID_INDEX32 is meaningful.
 * Closest-hit ties (equal t) resolve to the lowest (instance, primitive). */
int  s2_trace(S2Context* ctx, const S2Ray* rays, uint32_t count, int anyhit, S2Hit* hits, int on_device);
/* Same query with per-ray node/triangle fetch counts (uint32 pairs, device or host as above). */
int  s2_trace_counted(S2Context* ctx, const S2Ray* rays, uint32_t count, int anyhit, S2Hit* hits,
                      uint32_t* fetch_counts, int on_device);

/* ---- rendering (replaces TestRenderer::render) ------------------------------------------- */
int  s2_render(S2Context* ctx, const S2View* view, const S2RenderParams* params,
               const S2Aovs* out, int out_on_host, S2RenderStats* stats_out);

/* Batched rendering: `view_count` views (up to 255, any resolutions) in one call, each with
 * params->spp samples.  Paths of all views stream through one queue of params->wave_paths
 * entries (0 = 32M): before every bounce the queue is topped up with new camera paths, so
 * launches stay full however unevenly paths end (Russian roulette, escapes); each pair of bounces
 * is a captured CUDA graph replayed until the device reports all paths done.  Radiance
 * accumulates in 2^-24 fixed point (order-independent integer sums: deterministic).  `outs` has
 * one S2Aovs per view (host or device pointers per `out_on_host`).  S2_FLAG_ACCUMULATE adds to the
 * previous call with the same view extents.  Results equal s2_render's per view up to the
 * fixed-point rounding. */
int  s2_render_views(S2Context* ctx, const S2View* views, uint32_t view_count, const S2RenderParams* params,
                     const S2Aovs* outs, int out_on_host, S2RenderStats* stats_out);

/* Defaults as in the reference (TestRenderer.cpp:38-43, VCM.cpp:39-40). */
void s2_default_render_params(S2RenderParams* p);

/* Failure-detection test (diagnostic; no counterpart in the reference): arms the next launch of the
 * radiance cache's inference kernel (s2_cache_query, or the cache step of a render) to wait on its
 * first-layer mbarrier without issuing that layer's MMA or commit -- an arrival that never comes --
 * with each of its bounded waits limited to `polls` polls (1..2^20).  The launch gives up, frees
 * its TMEM and returns; the call reports S2_ERR_TIMEOUT and the context stays usable.  One-shot. */
int  s2_inject_wait_timeout(S2Context* ctx, uint32_t polls);

/* ---- device math check (diagnostic) ------------------------------------------------------
 * Evaluates one of the device math functions of the path tracer on n entries, for checks against
 * the reference's own shader functions (src/Shaders/common/rng.hlsli, common.hlsli,
 * microfacet.hlsli).  Host arrays: `in` holds 8 doubles per entry, `out` receives 9 per entry
 * (unsigned integers as exact doubles; float arguments are rounded to float first).
 *   0 xxhash32 (u -> h)                    1 pcg (u -> h)
 *   2 pcg4d (u4 -> u4)                     3 RandomSampler: first nextFloat() of state
 *                                            (px, py, seed, offset) -> 4 floats
 *   4 packNormal (xyz -> packed)           5 unpackNormal (packed -> xyz)
 *   6 GTR1 (n.h, alpha)                    7 GTR2 anisotropic (h.xyz, ax, ay)
 *   8 smith_masking_gtr2 (v.xyz, ax, ay)   9 smith_masking_gtr1 (v.xyz)
 *  10 sample_visible_normals (in.xyz, ax, ay, u1, u2 -> h.xyz)
 *  11 schlick_fresnel (F0, cos)           12 fresnel_dielectric (n.i, eta)
 *  13 sampleConcentricDisc (u1, u2 -> xy) 14 sampleCosHemisphere (u1, u2 -> xyz)
 *  15 sampleUniformSphere (u1, u2 -> xyz) 16 sampleUniformTriangle (u1, u2 -> b1, b2)
 *  17 makeOrthonormal (n.xyz -> rows t, b, n) */
int  s2_device_math(S2Context* ctx, int function_id, const double* in, uint32_t n, double* out);

/* ---- allocation-free rendering ----------------------------------------------------------
 * No counterpart in the reference.  For callers that may not allocate device memory while they
 * render (a host application that owns the GPU's memory budget and forbids cudaMalloc/cudaFree,
 * which also synchronise the device, once its frame loop runs; a plugin limited to the buffers
 * its host hands it).  Same kernels and results as s2_render, but the path queues, hit records,
 * shadow rays, accumulators and counters live in one 64 MiB file-scope device array of the
 * library, held on every GPU that loads it until the process exits, and radiance accumulates in
 * the caller's output.  Allocates nothing.
 *   - `out` holds DEVICE pointers; out->radiance is required; other AOVs may be NULL.
 *   - Views above 322,603 pixels (64 MiB less a 4 KiB header and 13 x 256 bytes of stream
 *     alignment, / 208 bytes per path; e.g. 512x512 fits, 1920x1080 does not) are rejected with
 *     S2_ERR_INVALID.  S2_FLAG_ACCUMULATE and S2_FLAG_PROFILE_KERNELS are rejected, and so are
 *     the modes with buffers of their own (ReSTIR reuse, radiance cache, light tracing:
 *     S2_ERR_UNSUPPORTED).
 *   - The first call on a device looks up the array's address; make it before any stream capture.
 *   - Calls share the array: calls whose GPU work overlaps race; serialise them. */
int  s2_render_noalloc(S2Context* ctx, const S2View* view, const S2RenderParams* params,
                       const S2Aovs* out, S2RenderStats* stats_out);

/* Tuning of the wavefront renderer (no counterpart in the reference).  Zero fields select the
 * defaults.  s2_autotune measures candidates on the caller's scene, view and parameters and
 * applies the fastest; s2_set_tuning applies a stored result (stratum2_b200/autotune.py keeps them
 * as JSON keyed by GPU and workload). */
#define S2_SHADE_ORDER_MATERIAL 0u
#define S2_SHADE_ORDER_QUEUE 1u
#define S2_TRACE_ORDER_QUEUE 0u
#define S2_TRACE_ORDER_COHERENT 1u
#define S2_SHADE_RECORDS_ON 0u
#define S2_SHADE_RECORDS_OFF 1u
#define S2_SHADOW_MERGE_ON    0u
#define S2_SHADOW_MERGE_OFF   1u

typedef struct S2Tuning {
    uint32_t wave_paths;          /* paths per wave when S2RenderParams.wave_paths is 0 (0 = 2^26) */
    uint32_t trav_tris_per_step;  /* triangle tests per triangle step of the traversal (0 = 4) */
    uint32_t trav_vote8;          /* triangle step when vote8/8 of the busy lanes have triangles (0 = 4) */
    uint32_t refill_min;          /* traversal lanes refilled once this many are idle (0 = 8) */
    uint32_t shade_order;         /* S2_SHADE_ORDER_MATERIAL (0, default): counting-sort the path queue by
                                     hit material before shading; S2_SHADE_ORDER_QUEUE (1): shade in queue
                                     order.  Images are bit-identical either way. */
    uint32_t trace_order;         /* S2_TRACE_ORDER_QUEUE (0, default): trace continuation rays in queue
                                     order; S2_TRACE_ORDER_COHERENT (1): counting-sort them by origin cell
                                     and direction octant first.  Images are bit-identical either way. */
    uint32_t shade_records;       /* S2_SHADE_RECORDS_ON (0, default): hits on meshes without texture
                                     coordinates or normals read a 64-byte shading record baked per BVH
                                     triangle at s2_build_bvh; S2_SHADE_RECORDS_OFF (1): gather through
                                     the instance and vertex buffers as the reference does.  Images are
                                     bit-identical either way. */
    uint32_t shadow_merge;        /* S2_SHADOW_MERGE_ON (0, default): a bounce's shadow rays are traced by
                                     the next bounce's traversal launch, after its closest hits (one
                                     persistent launch for both queues; not with the radiance cache);
                                     S2_SHADOW_MERGE_OFF (1): a separate any-hit launch after every shade.
                                     Images are bit-identical either way. */
} S2Tuning;

int  s2_set_tuning(S2Context* ctx, const S2Tuning* tuning);
int  s2_get_tuning(S2Context* ctx, S2Tuning* tuning);
/* Coordinate search over wave size, triangle batch, vote, refill threshold, shading order, trace order and
 * shadow merging: every candidate
 * renders `params` (its spp; frame seeds advance per trial) and the highest ray throughput wins.
 * The result is applied to `ctx` and written to `out` (may be NULL); `trials_out` (may be NULL)
 * receives the number of timed renders. */
int  s2_autotune(S2Context* ctx, const S2View* view, const S2RenderParams* params, S2Tuning* out,
                 uint32_t* trials_out);

/* Replaces the texels of uploaded image `index` (same width, height and channel count as at
 * s2_scene_upload; host or device pointer).  An environment image gets its sampling tables rebuilt.
 * The alpha-test flags baked into the BVH at s2_build_bvh are not recomputed. */
int  s2_update_image(S2Context* ctx, uint32_t index, const float* texels, int on_device);

/* Texture repack of a glTF metallic-roughness material on the device: the reference's from_gltf_pbr
 * pass (src/Shaders/kernels/convert_material.slang:33-69, dispatched by makeMetallicRoughnessMaterial,
 * src/App/Scene.cpp:195-208, for the textures load_gltf.cpp:92-128 passes it).  Sources are RGBA8
 * texels of one width x height (NULL = absent, read as 1): the base colour (sRGB rgb, linear alpha),
 * the metallic-roughness texture (linear; metallic b, roughness g) and the emission (sRGB rgb); at
 * least one is required.  Per texel the PackedMaterialData of those values is written as the four
 * packed words' images, float4 each (byte / 255): packed[0] base colour + specular 1, packed[1]
 * emission / its largest channel + sheen 1, packed[2] metallic, roughness, anisotropic 1,
 * subsurface 1, packed[3] clearcoat, clearcoat gloss, transmission and eta all 1.  alpha_mask (may
 * be NULL; needs the base colour) receives the base colour's alpha as one float per texel, and
 * *min_alpha the smallest 8-bit alpha below 255 (255 when every texel is opaque or there is no base
 * colour).  on_device: all pointers but min_alpha are device pointers (sources 4-byte, packed
 * images 16-byte aligned); else host pointers. */
int  s2_repack_metallic_roughness(S2Context* ctx, uint32_t width, uint32_t height, const uint8_t* base_rgba8,
                                  const uint8_t* metallic_roughness_rgba8, const uint8_t* emission_rgba8,
                                  float* const* packed, float* alpha_mask, uint32_t* min_alpha, int on_device);

/* ---------------------------------------------------------------- differentiable rendering
 * No counterpart in the reference.  The same path tracer as s2_render (NEE + MIS, Russian
 * roulette, path-length gates, the same random numbers per pixel and sample) with textured material
 * parameters kept in f32 instead of being re-quantised to 8 bits, so the image is differentiable in
 * the texels.  Not supported: ReSTIR, the radiance cache, accumulation, profiling flags, AOVs. */
/* radiance: float4 per pixel (mean * 2^exposure, w = 1), host (out_on_host) or device. */
int  s2_render_diff(S2Context* ctx, const S2View* view, const S2RenderParams* params, float* radiance,
                    int out_on_host, S2RenderStats* stats_out);
/* Adjoint path replay: d_images[k] (float4 per texel of image k, or NULL to skip) receives the
 * gradient of sum(d_radiance * radiance) with respect to image k's texels, where radiance is the
 * s2_render_diff image for the same view and params.  Every path is replayed twice from its seed:
 * once for its radiance, once to push the adjoint through its vertices.  Sampling pdfs, MIS weights
 * and Russian roulette are held constant.  Gradients reach base-colour textures (rgb), packed[2]
 * textures (roughness channel, y) and the environment image (rgb).  on_host applies to d_radiance
 * and d_images alike. */
int  s2_render_adjoint(S2Context* ctx, const S2View* view, const S2RenderParams* params, const float* d_radiance,
                       int on_host, float* const* d_images, S2RenderStats* stats_out);

/* ---------------------------------------------------------------- learned radiance cache
 * No counterpart in the reference.  A multiresolution hash-grid encoding of world-space position
 * (16 levels x 2 features, 2^log2_table entries per level, resolutions geometric from
 * base_resolution to max_resolution over the cache box) feeding a 32 -> 64 -> 64 -> 3 ReLU MLP
 * without biases (6,336 weights).  f16 parameters on the device with f32 master copies; inference
 * and training run on the tensor cores (f16 operands, f32 accumulation).  Parameter order of the
 * weights: W1 (64 x 32, row = output), W2 (64 x 64), W3 (3 x 64); the table: [level][entry][2]. */
#define S2_CACHE_WEIGHTS 6336
#define S2_CACHE_LEVELS  16

typedef struct S2CacheParams {
    float box_min[3], box_max[3];   /* encoding domain; box_min >= box_max: the scene bounding sphere's box */
    uint32_t log2_table;            /* default 19 */
    uint32_t base_resolution;       /* default 16 */
    uint32_t max_resolution;        /* default 2048 */
    float learning_rate;            /* Adam, default 1e-2 */
    float beta1, beta2, epsilon;    /* default 0.9, 0.99, 1e-15 */
    uint32_t seed;                  /* parameter initialisation */
    uint32_t reserved[6];
} S2CacheParams;                    /* 80 B */

void s2_cache_default_params(S2CacheParams* p);
/* (Re)creates the cache with freshly initialised parameters (table U(-1e-4, 1e-4), weights
 * U(+-sqrt(6 / (fan_in + fan_out))) from `seed`). */
int  s2_cache_init(S2Context* ctx, const S2CacheParams* params);
/* Copies the f32 parameters out / in (weights: S2_CACHE_WEIGHTS floats; table: 16 * 2^log2_table
 * * 2 floats; either pointer may be NULL).  Setting resets the optimiser state. */
int  s2_cache_get_params(S2Context* ctx, float* weights, float* table);
int  s2_cache_set_params(S2Context* ctx, const float* weights, const float* table);
/* Evaluates the cache at n positions: positions and radiance are float4 per entry (xyz used). */
int  s2_cache_query(S2Context* ctx, const float* positions, uint32_t n, float* radiance, int on_device);
/* One optimiser step (Adam on the f32 masters, then refreshed f16 copies; table entries no record
 * touched keep their parameters and moments, as in lazy Adam) on n records: float4
 * positions and float4 target radiances.  Loss per record: sum_c (y_c - t_c)^2 / (y_c^2 + 0.01) / 3
 * with the denominator held constant; `loss` (may be NULL) receives its mean over the records. */
int  s2_cache_train(S2Context* ctx, const float* positions, const float* targets, uint32_t n, float* loss,
                    int on_device);
/* The gradients of the mean loss over n records without an optimiser step (host outputs: weights
 * S2_CACHE_WEIGHTS floats, table 16 * 2^log2_table * 2 floats; either may be NULL). */
int  s2_cache_gradients(S2Context* ctx, const float* positions, const float* targets, uint32_t n,
                        float* grad_weights, float* grad_table, float* loss, int on_device);

/* ---- post-processing (replaces the Denoiser's temporal accumulation and the Tonemapper) ---- */
/* Temporal accumulation (src/Shaders/kernels/svgf/temporal_accumulation.slang:34-129, driven by
 * Denoiser.cpp:121-201): a running average of the frames rendered by s2_render, reprojected
 * through the prev_uv AOV with per-tap instance / normal / depth rejection.  The context keeps the
 * history (previous accumulated colour and moments, visibility and depth). */
#define S2_TEMPORAL_REPROJECT          (1u << 0)  /* gReprojection (default on, Denoiser.cpp:24) */
#define S2_TEMPORAL_CHECK_NORMAL       (1u << 1)  /* gCheckNormal (default on) */
#define S2_TEMPORAL_CHECK_DEPTH        (1u << 2)  /* gCheckDepth (default on) */
#define S2_TEMPORAL_DEMODULATE_ALBEDO  (1u << 3)  /* gDemodulateAlbedo */
#define S2_TEMPORAL_SHADOW_HYSTERESIS  (1u << 4)  /* gShadowHysteresis */
#define S2_TEMPORAL_RESET              (1u << 5)  /* drop the history first (mResetAccumulation) */

typedef struct S2TemporalParams {
    uint32_t flags;                  /* S2_TEMPORAL_* */
    uint32_t history_limit;          /* mHistoryLimit: cap of the accumulated count, 0 = none */
    float shadow_preserve_offset;    /* mShadowPreserveOffset (0.1) */
    float shadow_preserve_scale;     /* mShadowPreserveScale (1) */
} S2TemporalParams;

/* The reference's defaults: reprojection with normal and depth checks, no history limit. */
void s2_default_temporal_params(S2TemporalParams* p);
/* One frame: `frame` holds the DEVICE AOVs of one s2_render call of `view` (radiance and, with
 * reprojection, visibility, depth and prev_uv; albedo when demodulating).  instance_index_map
 * (device, may be NULL = identity) maps this frame's instance ids to the previous frame's
 * (mInstanceIndexMap).  Writes the accumulated colour (float4: rgb, sample count) and, when not
 * NULL, the luminance moments (float2) to DEVICE buffers of the view's extent.  The first call, a
 * reset or a change of extent starts a new history. */
int  s2_temporal_accumulate(S2Context* ctx, const S2View* view, const S2TemporalParams* params, const S2Aovs* frame,
                            const uint32_t* instance_index_map, float* accum_color, float* accum_moments);

/* SVGF filter over the context's accumulation history (Denoiser.cpp:202-241:
 * svgf/estimate_variance.slang, then `iterations` passes of svgf/atrous.slang with step 2^i).
 * Call after s2_temporal_accumulate for the same view and frame. */
#define S2_SVGF_KERNEL_ATROUS            0u  /* FilterKernelType (compat/filter_type.h) */
#define S2_SVGF_KERNEL_BOX3              1u  /* the reference's default */
#define S2_SVGF_KERNEL_BOX5              2u
#define S2_SVGF_KERNEL_SUBSAMPLED        3u
#define S2_SVGF_KERNEL_BOX3_SUBSAMPLED   4u
#define S2_SVGF_KERNEL_BOX5_SUBSAMPLED   5u

typedef struct S2SvgfParams {
    uint32_t iterations;             /* mAtrousIterations (1..16) */
    uint32_t kernel;                 /* S2_SVGF_KERNEL_* */
    uint32_t history_tap;            /* mHistoryTap: after this iteration (1-based) the filtered colour
                                        replaces the history's colour (0 = never) */
    uint32_t flags;                  /* S2_TEMPORAL_CHECK_NORMAL / S2_TEMPORAL_CHECK_DEPTH edge stops */
    uint32_t history_limit;          /* mHistoryLimit: histories shorter than it get a spatial
                                        variance estimate (0: never, as in the reference default) */
    float variance_boost_length;     /* mVarianceBoostLength (4) */
    float sigma_luminance_boost;     /* mSigmaLuminanceBoost (3) */
    uint32_t reserved;
} S2SvgfParams;

/* The reference's Denoiser defaults with 5 iterations (mAtrousIterations is 0 = off there). */
void s2_default_svgf_params(S2SvgfParams* p);
/* `frame` holds the same DEVICE visibility and depth AOVs as the accumulation call; output is a
 * DEVICE float4 image of the view's extent (rgb filtered, a = filtered variance). */
int  s2_svgf_filter(S2Context* ctx, const S2View* view, const S2SvgfParams* params, const S2Aovs* frame,
                    const uint32_t* instance_index_map, float* output);

/* Tonemapping (src/Shaders/kernels/tonemap.slang:113-192, Tonemapper.cpp:49-97): maximum reduce,
 * radiance x 2^exposure, one operator, optional gamma.  Modes follow TonemapMode
 * (compat/tonemap.h). */
#define S2_TONEMAP_RAW                       0u
#define S2_TONEMAP_REINHARD                  1u
#define S2_TONEMAP_REINHARD_EXTENDED         2u
#define S2_TONEMAP_REINHARD_LUMINANCE        3u
#define S2_TONEMAP_REINHARD_LUMINANCE_EXT    4u
#define S2_TONEMAP_UNCHARTED2                5u
#define S2_TONEMAP_FILMIC                    6u
#define S2_TONEMAP_ACES                      7u
#define S2_TONEMAP_ACES_APPROX               8u
#define S2_TONEMAP_VIRIDIS_R                 9u
#define S2_TONEMAP_VIRIDIS_LENGTH_RGB       10u
#define S2_TONEMAP_GAMMA            (1u << 0)  /* standard sRGB encoding of the result */
#define S2_TONEMAP_GAMMA_REFERENCE  (1u << 1)  /* the reference's rgbToSrgb (compat/common.h:88-93),
                                                  pow(1.055 x, 1/2.4) - 0.055, which is not sRGB:
                                                  compatibility mode */

typedef struct S2TonemapParams {
    uint32_t mode;                   /* S2_TONEMAP_RAW .. S2_TONEMAP_VIRIDIS_LENGTH_RGB */
    float exposure;                  /* mExposure: radiance x 2^exposure */
    uint32_t flags;                  /* S2_TONEMAP_GAMMA / S2_TONEMAP_GAMMA_REFERENCE */
    uint32_t reserved;
} S2TonemapParams;

/* DEVICE float4 images of width x height; `albedo` (may be NULL) modulates the input
 * (gModulateAlbedo: radiance x (0.01 + albedo), and albedo x radiance in the maximum). */
int  s2_tonemap(S2Context* ctx, uint32_t width, uint32_t height, const S2TonemapParams* params, const float* input,
                const float* albedo, float* output);

/* ---------------------------------------------------------------- vertex connection and merging
 * Replaces the reference's VCM renderer (VCM.cpp:370-620, vcm.slang:880-1238: SmallVCM's
 * bidirectional techniques with the MIS quantities dVCM / dVC / dVM).  Each iteration traces
 * n_light = max(1, pixels x light_path_fraction) light subpaths, then one camera path per pixel.
 * Camera samples are jittered over their pixel (the reference uses pixel centres), so camera paths
 * and camera connections estimate the same box-filtered image.  The environment is black and never
 * sampled, as in the reference (GetBackgroundRadiance returns zero radiance); only area lights
 * emit.  The merge radius of iteration i is max(1e-7, merge_radius_factor x scene radius /
 * (i + 1)^(0.5 (1 - merge_radius_alpha))), i = first_iteration + the iteration's index
 * (VCM.cpp:454-457). */
#define S2_VCM_PATH_TRACE   0u  /* VcmAlgorithmType (compat/vcm.h:103-132) */
#define S2_VCM_LIGHT_TRACE  1u
#define S2_VCM_PPM          2u
#define S2_VCM_BPM          3u
#define S2_VCM_BPT          4u
#define S2_VCM_VCM          5u
#define S2_VCM_FLAG_LIGHT_VERTEX_CACHE  (1u << 0)  /* BPT: one connection to a random cached light
                                                      vertex (mUseLightVertexCache, the reference's
                                                      default) instead of all vertices of one subpath */
#define S2_VCM_FLAG_DEBUG_PATHS         (1u << 1)  /* gDebugPaths: keep only the technique with
                                                      debug_camera_vertices / debug_light_vertices */
#define S2_VCM_FLAG_DEBUG_UNWEIGHTED    (1u << 2)  /* with DEBUG_PATHS and not gDebugPathWeights: every
                                                      MIS weight 1 */
#define S2_VCM_FLAG_DI_RIS              (1u << 3)  /* gDIReservoirFlags eRIS: the direct illumination of
                                                      camera vertices resamples di_candidates light
                                                      samples by lum(Le) |cos| G and traces one shadow
                                                      ray for the chosen one (vcm.slang:343-366) */
#define S2_VCM_FLAG_LVC_RIS             (1u << 5)  /* with LIGHT_VERTEX_CACHE, gLVCReservoirFlags eRIS:
                                                      each camera vertex resamples lvc_candidates
                                                      random cached light vertices by the luminance
                                                      of their connection and traces one shadow ray
                                                      (vcm.slang:568-736) */
#define S2_VCM_FLAG_LVC_REUSE           (1u << 6)  /* with LVC_RIS, eReuse: each camera vertex also
                                                      resamples an LVC reservoir of the previous
                                                      iteration (or call) found in a world-space hash
                                                      grid near it, and stores its own with the light
                                                      vertex by value (vcm.slang:633-726) */
#define S2_VCM_FLAG_DI_REUSE            (1u << 4)  /* with DI_RIS, eReuse: each camera vertex also
                                                      resamples a reservoir of the previous iteration
                                                      (or call) found in a world-space hash grid near it
                                                      and stores its own (vcm.slang:296-340, 368-386);
                                                      not with PPM or light tracing */

typedef struct S2VcmParams {
    uint32_t algorithm;              /* S2_VCM_PATH_TRACE .. S2_VCM_VCM (default S2_VCM_BPT, VCM.hpp:66) */
    uint32_t min_path_length;        /* mMinPathLength (default 0) */
    uint32_t max_path_length;        /* mMaxPathLength (default 6), 1..64 */
    uint32_t iterations;             /* light pass + camera pass per iteration; the image is their mean */
    uint32_t frame_seed;             /* mRandomSeed of the first iteration (+1 per iteration) */
    uint32_t first_iteration;        /* index of the first iteration in the merge-radius schedule */
    uint32_t flags;                  /* S2_FLAG_LAMBERTIAN, PCG32, NO_RR, SHADING_NORMALS_OFF,
                                        ALPHA_TEST_OFF, NORMAL_MAPS_OFF, LIGHT_POWER_PICK */
    uint32_t vcm_flags;              /* S2_VCM_FLAG_* */
    float light_path_fraction;       /* mLightPathPercent (default 1) */
    float merge_radius_factor;       /* mVmRadiusFactor (default 0.025) */
    float merge_radius_alpha;        /* mVmRadiusAlpha (default 0.01) */
    float exposure;                  /* output x 2^exposure */
    uint16_t debug_camera_vertices;  /* mDebugPathLengths (compat/vcm.h:49-55) */
    uint16_t debug_light_vertices;
    uint32_t di_candidates;          /* mDIReservoirSampleCount (default 32, VCM.cpp:33), 1..1024 */
    float di_max_m;                  /* mDIReservoirMaxM (default 3, VCM.cpp:34): stored M is capped
                                        at di_max_m x di_candidates */
    uint32_t lvc_candidates;         /* mLVCReservoirSampleCount (default 8, VCM.cpp:35), 1..1024 */
    float lvc_max_m;                 /* mLVCReservoirMaxM (default 3, VCM.cpp:36): stored M is capped
                                        at lvc_max_m x lvc_candidates */
} S2VcmParams;

void s2_default_vcm_params(S2VcmParams* p);
/* One call renders `iterations` iterations of the view.  AOVs (albedo 0 on a miss, as in the VCM
 * renderer) come from the first iteration's camera paths.  stats_out: extension and shadow rays of
 * both passes, paths = pixels x iterations.  S2_ERR_UNSUPPORTED for flags outside the list above or
 * the light vertex cache with an algorithm other than BPT. */
int  s2_render_vcm(S2Context* ctx, const S2View* view, const S2VcmParams* params, const S2Aovs* out, int out_on_host,
                   S2RenderStats* stats_out);

#ifdef __cplusplus
}
#endif

#endif  /* STRATUM2_H_ */
