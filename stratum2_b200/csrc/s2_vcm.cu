// Vertex connection and merging entry points (s2_render_vcm, s2_default_vcm_params), replacing the
// reference's VCM renderer (VCM.cpp:370-620).  Kernels in s2_vcm.cuh.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "s2_context.h"

// The renderer's device code, compiled here with internal linkage (inside an unnamed namespace,
// its namespace renamed) so the header-defined kernels do not collide with s2_render.cu's.
#define s2 s2_vcm_impl
namespace {
#include "s2_vcm.cuh"
}  // namespace
#undef s2
namespace vk = s2_vcm_impl;
using s2::DevBuf;
using s2::check_cuda;
using s2::dev_alloc;
using s2::free_bufs;
using s2::set_error;

namespace {

constexpr uint32_t kVcmRenderFlags = S2_FLAG_LAMBERTIAN | S2_FLAG_PCG32 | S2_FLAG_NO_RR | S2_FLAG_SHADING_NORMALS_OFF |
                                     S2_FLAG_ALPHA_TEST_OFF | S2_FLAG_NORMAL_MAPS_OFF | S2_FLAG_LIGHT_POWER_PICK;
constexpr uint32_t kVcmOwnFlags = S2_VCM_FLAG_LIGHT_VERTEX_CACHE | S2_VCM_FLAG_DEBUG_PATHS | S2_VCM_FLAG_DEBUG_UNWEIGHTED |
                                   S2_VCM_FLAG_DI_RIS | S2_VCM_FLAG_DI_REUSE | S2_VCM_FLAG_LVC_RIS |
                                   S2_VCM_FLAG_LVC_REUSE;

void invert_affine(const float* m, float* out) {
    // inverse of a row-major 3x4 rigid (or scaled) transform
    const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
    const double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
    const double det = a * A + b * B + c * C;
    const double inv[9] = {A / det, -(b * i - c * h) / det, (b * f - c * e) / det,
                           B / det, (a * i - c * g) / det, -(a * f - c * d) / det,
                           C / det, -(a * h - b * g) / det, (a * e - b * d) / det};
    for (int r = 0; r < 3; ++r) {
        out[4 * r + 0] = (float)inv[3 * r + 0];
        out[4 * r + 1] = (float)inv[3 * r + 1];
        out[4 * r + 2] = (float)inv[3 * r + 2];
        out[4 * r + 3] = (float)-(inv[3 * r + 0] * m[3] + inv[3 * r + 1] * m[7] + inv[3 * r + 2] * m[11]);
    }
}

// The world-space grids of the direct-illumination and light-vertex-cache reservoirs (GpuHashGrid,
// src/App/GpuHashGrid.cpp:17-111, as the path tracer's reuse grids): appended to by one iteration's
// camera pass, read by the next one's.  An LVC grid keeps its 128-byte records in `wide`, at the
// data index of each record's sort key.
struct DiGrid {
    std::vector<DevBuf> bufs;
    HashGridDev g{};
    void* wide = nullptr;
    size_t wide_bytes = 0;
    unsigned long long *keys_in = nullptr, *keys_out = nullptr;
    uint32_t* vals_in = nullptr;
    void* sort_tmp = nullptr;
    size_t sort_bytes = 0;
    int end_bit = 64;
};

// `fresh` (optional) is set when the grid was (re)allocated: its buffers then hold no reservoirs.
int ensure_di_grid(S2Context* ctx, DiGrid& G, uint32_t cells, uint32_t size, size_t wide_bytes = 0, bool* fresh = nullptr) {
    if (G.g.checksums && G.g.cell_count == cells && G.g.max_size >= size && G.wide_bytes == wide_bytes) return S2_OK;
    if (fresh) *fresh = true;
    free_bufs(G.bufs);
    G.g = HashGridDev{};
    G.wide = nullptr;
    G.wide_bytes = 0;
    HashGridDev g{};
    auto al = [&](size_t bytes) { return dev_alloc(ctx, G.bufs, bytes); };
    g.checksums = (uint32_t*)al(sizeof(uint32_t) * cells);
    g.cell_counters = (uint32_t*)al(sizeof(uint32_t) * cells);
    g.other = (uint32_t*)al(sizeof(uint32_t) * 4);
    g.append_indices = (uint2*)al(sizeof(uint2) * size);
    g.data = (ReservoirRecord*)al(sizeof(ReservoirRecord) * size);
    g.indices = (uint32_t*)al(sizeof(uint32_t) * cells);
    g.data_indices = (uint32_t*)al(sizeof(uint32_t) * size);
    G.keys_in = (unsigned long long*)al(sizeof(unsigned long long) * size);
    G.keys_out = (unsigned long long*)al(sizeof(unsigned long long) * size);
    G.vals_in = (uint32_t*)al(sizeof(uint32_t) * size);
    int cell_bits = 1;  // keys: cell above a 32-bit content hash (unused slots take cell `cells`)
    while (cell_bits < 32 && (1ull << cell_bits) <= cells) ++cell_bits;
    G.end_bit = 32 + cell_bits;
    G.sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, G.sort_bytes, G.keys_in, G.keys_out, G.vals_in, g.data_indices, (int)size, 0,
                                    G.end_bit, ctx->stream);
    G.sort_tmp = al(std::max<size_t>(G.sort_bytes, 16));
    if (wide_bytes) G.wide = al(wide_bytes * size);
    for (auto& b : G.bufs) if (!b.ptr) { free_bufs(G.bufs); return S2_ERR_OOM; }
    if (G.bufs.size() != (wide_bytes ? 12u : 11u)) { free_bufs(G.bufs); return S2_ERR_OOM; }
    G.wide_bytes = wide_bytes;
    g.cell_count = cells;
    g.max_size = size;
    G.g = g;
    return S2_OK;
}

// Cell offsets by a scan, records sorted by (cell, content); returns the launches issued.
uint32_t build_di_grid(const DiGrid& G, cudaStream_t s) {
    const HashGridDev& g = G.g;
    k_hg_scan<<<1, kHgScanThreads, 0, s>>>(g);
    k_hg_keys<<<(g.max_size + 255) / 256, 256, 0, s>>>(g, G.keys_in, G.vals_in);
    size_t bytes = G.sort_bytes;
    cub::DeviceRadixSort::SortPairs(G.sort_tmp, bytes, G.keys_in, G.keys_out, G.vals_in, g.data_indices, (int)g.max_size, 0,
                                    G.end_bit, s);
    return 3;
}

template <bool LAMBERT>
void launch_light(const vk::VcmArgs& A, cudaStream_t s) {
    const uint32_t blocks = std::min<uint32_t>((A.n_light + 127) / 128, 148u * 8u);
    vk::k_vcm_light<LAMBERT><<<blocks, 128, 0, s>>>(A);
}
template <bool LAMBERT>
void launch_camera(const vk::VcmArgs& A, cudaStream_t s) {
    if (A.lvc_m) vk::k_vcm_camera<LAMBERT, true><<<(A.pixels + 127) / 128, 128, 0, s>>>(A);
    else vk::k_vcm_camera<LAMBERT, false><<<(A.pixels + 127) / 128, 128, 0, s>>>(A);
}

}  // namespace

namespace s2 {
// Kept in the context between calls: the reservoir grids of the last iteration, so that a call's
// first iteration reuses the previous call's reservoirs (the reference's frame-to-frame reuse).
struct VcmState {
    DiGrid grid[2];
    uint32_t cur = 0;
    bool prev_valid = false;
    DiGrid lvc_grid[2];  // the light-vertex-cache reservoirs, likewise
    uint32_t lvc_cur = 0;
    bool lvc_prev_valid = false;
};
void destroy_vcm_state(S2Context* ctx) {
    if (!ctx || !ctx->vcm) return;
    for (auto& g : ctx->vcm->grid) free_bufs(g.bufs);
    for (auto& g : ctx->vcm->lvc_grid) free_bufs(g.bufs);
    delete ctx->vcm;
    ctx->vcm = nullptr;
}
}  // namespace s2

extern "C" void s2_default_vcm_params(S2VcmParams* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->algorithm = S2_VCM_BPT;                       // VCM.hpp:66
    p->min_path_length = 0;                          // VCM.cpp:29-30
    p->max_path_length = 6;
    p->iterations = 1;
    p->vcm_flags = S2_VCM_FLAG_LIGHT_VERTEX_CACHE;   // mUseLightVertexCache = true (VCM.hpp:53)
    p->light_path_fraction = 1.f;                    // VCM.hpp:67
    p->merge_radius_factor = 0.025f;                 // VCM.hpp:59-60
    p->merge_radius_alpha = 0.01f;
    p->di_candidates = 32;                           // VCM.cpp:33-35
    p->di_max_m = 3.f;
    p->lvc_candidates = 8;
    p->lvc_max_m = 3.f;
}

extern "C" int s2_render_vcm(S2Context* ctx, const S2View* view, const S2VcmParams* prm, const S2Aovs* out, int out_on_host,
                             S2RenderStats* stats_out) {
    if (!ctx) return S2_ERR_INVALID;
    if (!view || !prm) return set_error(ctx, S2_ERR_INVALID, "view and params are required");
    if (!ctx->has_bvh) return set_error(ctx, S2_ERR_NO_SCENE, "s2_render_vcm before s2_scene_upload + s2_build_bvh");
    const int W = view->image_max[0] - view->image_min[0], H = view->image_max[1] - view->image_min[1];
    if (W <= 0 || H <= 0 || (int64_t)W * H > (1ll << 26)) return set_error(ctx, S2_ERR_INVALID, "invalid view extent");
    if (prm->algorithm > S2_VCM_VCM) return set_error(ctx, S2_ERR_INVALID, "unknown VCM algorithm");
    if (prm->max_path_length < 1 || prm->max_path_length > 64) return set_error(ctx, S2_ERR_INVALID, "max_path_length must be in 1..64");
    if (prm->iterations == 0) return set_error(ctx, S2_ERR_INVALID, "iterations must be >= 1");
    if (prm->flags & ~kVcmRenderFlags)
        return set_error(ctx, S2_ERR_UNSUPPORTED, "s2_render_vcm takes only the LAMBERTIAN, PCG32, NO_RR, SHADING_NORMALS_OFF, "
                                                  "ALPHA_TEST_OFF, NORMAL_MAPS_OFF and LIGHT_POWER_PICK flags");
    if (prm->vcm_flags & ~kVcmOwnFlags) return set_error(ctx, S2_ERR_INVALID, "unknown VCM flag");
    const uint32_t algo = prm->algorithm;
    const bool lvc = (prm->vcm_flags & S2_VCM_FLAG_LIGHT_VERTEX_CACHE) != 0;
    if (lvc && algo != S2_VCM_BPT) return set_error(ctx, S2_ERR_UNSUPPORTED, "the light vertex cache serves BPT only");
    if (!(prm->light_path_fraction > 0.f) || !std::isfinite(prm->light_path_fraction))
        return set_error(ctx, S2_ERR_INVALID, "light_path_fraction must be finite and > 0");
    const bool lvc_ris = (prm->vcm_flags & S2_VCM_FLAG_LVC_RIS) != 0;
    if (lvc_ris && !(prm->vcm_flags & S2_VCM_FLAG_LIGHT_VERTEX_CACHE))
        return set_error(ctx, S2_ERR_INVALID, "LVC_RIS needs LIGHT_VERTEX_CACHE");
    if (lvc_ris && (prm->lvc_candidates < 1 || prm->lvc_candidates > 1024))
        return set_error(ctx, S2_ERR_INVALID, "lvc_candidates must be in 1..1024");
    const bool lvc_reuse = (prm->vcm_flags & S2_VCM_FLAG_LVC_REUSE) != 0;
    if (lvc_reuse && !lvc_ris) return set_error(ctx, S2_ERR_INVALID, "LVC_REUSE needs LVC_RIS");
    if (lvc_reuse && !(prm->lvc_max_m > 0.f && std::isfinite(prm->lvc_max_m)))
        return set_error(ctx, S2_ERR_INVALID, "lvc_max_m must be finite and > 0");
    const bool di_ris = (prm->vcm_flags & S2_VCM_FLAG_DI_RIS) != 0;
    if ((prm->vcm_flags & S2_VCM_FLAG_DI_REUSE) && !di_ris) return set_error(ctx, S2_ERR_INVALID, "DI_REUSE needs DI_RIS");
    if (di_ris && (prm->di_candidates < 1 || prm->di_candidates > 1024))
        return set_error(ctx, S2_ERR_INVALID, "di_candidates must be in 1..1024");
    // the camera vertices' direct illumination exists in path tracing, BPT and VCM only
    const bool di_reuse = (prm->vcm_flags & S2_VCM_FLAG_DI_REUSE) && algo != S2_VCM_PPM && algo != S2_VCM_LIGHT_TRACE &&
                          algo != S2_VCM_BPM;
    if (di_reuse && !(prm->di_max_m > 0.f && std::isfinite(prm->di_max_m)))
        return set_error(ctx, S2_ERR_INVALID, "di_max_m must be finite and > 0");
    const bool use_vc = algo == S2_VCM_BPT || algo == S2_VCM_VCM;
    const bool use_vm = algo == S2_VCM_PPM || algo == S2_VCM_BPM || algo == S2_VCM_VCM;
    const float R = ctx->scene.scene_sphere.w;
    if (use_vm && (!(prm->merge_radius_factor > 0.f) || !std::isfinite(prm->merge_radius_factor) ||
                   !std::isfinite(prm->merge_radius_alpha) || !(R > 0.f)))
        return set_error(ctx, S2_ERR_INVALID, "merging needs merge_radius_factor > 0, a finite merge_radius_alpha and a "
                                              "scene bounding sphere");
    const uint32_t pixels = (uint32_t)W * (uint32_t)H;
    const double nl = std::floor((double)pixels * (double)prm->light_path_fraction);
    if (nl > (double)(1u << 28)) return set_error(ctx, S2_ERR_INVALID, "too many light subpaths (pixels x light_path_fraction)");
    const uint32_t n_light = (uint32_t)std::max(1.0, nl);
    const bool store = use_vc || use_vm;
    const uint64_t slots64 = store ? (uint64_t)n_light * (prm->max_path_length - 1) : 0;
    if (slots64 > 0x7fffffffull) return set_error(ctx, S2_ERR_INVALID, "light vertex storage exceeds 2^31 slots");
    const uint32_t slots = (uint32_t)slots64;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;

    vk::VcmArgs A;
    std::memset(&A, 0, sizeof(A));
    A.scene = ctx->scene;
    A.scene.env_address = 0xffffffffu;  // black environment (see the header)
    A.scene.env_sample_prob = 0.f;
    A.scene.light_power_pick = (prm->flags & S2_FLAG_LIGHT_POWER_PICK) ? 1u : 0u;
    A.scene.env_fp_on = (prm->flags & S2_FLAG_ENV_FOOTPRINT_PDF) ? 1u : 0u;
    std::memcpy(A.proj, view->projection, sizeof(A.proj));
    A.imin[0] = view->image_min[0]; A.imin[1] = view->image_min[1];
    A.imax[0] = view->image_max[0]; A.imax[1] = view->image_max[1];
    std::memcpy(A.cam, view->camera_to_world, sizeof(A.cam));
    std::memcpy(A.prev_inv, view->prev_world_to_camera, sizeof(A.prev_inv));
    invert_affine(view->camera_to_world, A.cam_inv);
    A.image_plane_dist = std::fabs((float)H) / (2.f * std::tan(view->projection[7] * 0.5f));
    A.width = (uint32_t)W; A.height = (uint32_t)H; A.pixels = pixels;
    A.n_light = n_light;
    A.min_len = prm->min_path_length;
    A.max_len = prm->max_path_length;
    A.flags = prm->flags;
    A.use_vc = use_vc; A.use_vm = use_vm; A.ppm = algo == S2_VCM_PPM;
    A.light_trace_only = algo == S2_VCM_LIGHT_TRACE; A.path_trace_only = algo == S2_VCM_PATH_TRACE;
    A.lvc = lvc;
    A.debug_paths = (prm->vcm_flags & S2_VCM_FLAG_DEBUG_PATHS) ? 1u : 0u;
    A.debug_unweighted = A.debug_paths && (prm->vcm_flags & S2_VCM_FLAG_DEBUG_UNWEIGHTED) ? 1u : 0u;
    A.debug_cam = prm->debug_camera_vertices;
    A.debug_light = prm->debug_light_vertices;
    A.lv_slots = slots;
    A.status = ctx->status_dev;
    A.di_ris = di_ris ? 1u : 0u;
    A.di_reuse = di_reuse ? 1u : 0u;
    A.di_m = prm->di_candidates;
    A.di_max_m = prm->di_max_m;
    A.lvc_m = lvc_ris ? prm->lvc_candidates : 0u;
    A.lvc_reuse = lvc_reuse ? 1u : 0u;
    A.lvc_max_m = prm->lvc_max_m;
    s2::VcmState* vs = nullptr;
    if (di_reuse || lvc_reuse) {
        if (!ctx->vcm) ctx->vcm = new (std::nothrow) s2::VcmState();
        vs = ctx->vcm;
        if (!vs) return set_error(ctx, S2_ERR_OOM, "VCM state allocation failed");
    }
    if (lvc_reuse) {
        // VCM.cpp:27, 491-500: as the DI grid, one record per camera vertex
        const uint32_t cells = 100000u;
        const uint32_t size = (uint32_t)std::min<uint64_t>((uint64_t)pixels * std::max(1u, prm->max_path_length - 1), 1u << 24);
        // a grid reallocated for a larger call holds no reservoirs: if it is the one the first
        // iteration would read, there is no history
        for (uint32_t k = 0; k < 2; ++k) {
            DiGrid& g = vs->lvc_grid[k];
            bool fresh = false;
            const int rc0 = ensure_di_grid(ctx, g, cells, size, sizeof(vk::LvcRecord), &fresh);
            if (fresh && k != vs->lvc_cur) vs->lvc_prev_valid = false;
            if (rc0 != S2_OK) { vs->lvc_prev_valid = false; return set_error(ctx, rc0, "LVC reservoir grid allocation failed"); }
            g.g.min_cell_size = 0.1f;
            g.g.cell_pixel_radius = 0.f;
            g.g.camera_position = make_float3(view->camera_to_world[3], view->camera_to_world[7], view->camera_to_world[11]);
            g.g.distance_scale = 0.f;
        }
    } else if (ctx->vcm) {
        ctx->vcm->lvc_prev_valid = false;  // a call without LVC reuse drops its grids
    }
    if (di_reuse) {
        // VCM.cpp:26, 490-499: 100,000 cells of at least 0.1, one record per camera vertex
        const uint32_t cells = 100000u;
        const uint32_t size = (uint32_t)std::min<uint64_t>((uint64_t)pixels * std::max(1u, prm->max_path_length - 1), 1u << 24);
        for (uint32_t k = 0; k < 2; ++k) {  // as for the LVC grids above
            DiGrid& g = vs->grid[k];
            bool fresh = false;
            const int rc0 = ensure_di_grid(ctx, g, cells, size, 0, &fresh);
            if (fresh && k != vs->cur) vs->prev_valid = false;
            if (rc0 != S2_OK) { vs->prev_valid = false; return set_error(ctx, rc0, "reservoir grid allocation failed"); }
            g.g.min_cell_size = 0.1f;
            g.g.cell_pixel_radius = 0.f;
            g.g.camera_position = make_float3(view->camera_to_world[3], view->camera_to_world[7], view->camera_to_world[11]);
            g.g.distance_scale = 0.f;  // tan(0): cells of the minimum size everywhere
        }
    } else if (ctx->vcm) {
        ctx->vcm->prev_valid = false;  // a call without reuse drops the grids (VCM.cpp:231-235)
    }

    std::vector<DevBuf> tmp;
    auto fail = [&](int code, const char* msg) { cudaStreamSynchronize(s); free_bufs(tmp); return set_error(ctx, code, msg); };
    A.image_fx = (unsigned long long*)dev_alloc(ctx, tmp, 32ull * pixels);
    A.counts = (unsigned long long*)dev_alloc(ctx, tmp, 4 * sizeof(unsigned long long));
    if (!A.image_fx || !A.counts) return fail(S2_ERR_OOM, "VCM accumulator allocation failed");
    unsigned int* lvc_count = (unsigned int*)(A.counts + 3);
    uint32_t grid_bits = 1;
    void* sort_tmp = nullptr;
    size_t sort_bytes = 0;
    uint32_t *keys_out = nullptr, *vals_out = nullptr;
    const bool sort = use_vm || lvc;
    if (store) {
        A.lv = (vk::LightVertex*)dev_alloc(ctx, tmp, sizeof(vk::LightVertex) * std::max<uint64_t>(slots, 1));
        A.lv_count = (uint32_t*)dev_alloc(ctx, tmp, sizeof(uint32_t) * n_light);
        if (!A.lv || !A.lv_count) return fail(S2_ERR_OOM, "light vertex allocation failed");
        cudaMemsetAsync(A.lv_count, 0, sizeof(uint32_t) * n_light, s);
    }
    if (sort && slots > 0) {
        if (use_vm) {
            while ((1ull << grid_bits) < slots && grid_bits < 30) grid_bits++;
            A.grid_mask = (1u << grid_bits) - 1u;
            A.grid_start = (uint32_t*)dev_alloc(ctx, tmp, sizeof(uint32_t) << grid_bits);
            A.grid_end = (uint32_t*)dev_alloc(ctx, tmp, sizeof(uint32_t) << grid_bits);
            if (!A.grid_start || !A.grid_end) return fail(S2_ERR_OOM, "merge grid allocation failed");
        }
        A.grid_key = (uint32_t*)dev_alloc(ctx, tmp, sizeof(uint32_t) * slots);
        A.grid_val = (uint32_t*)dev_alloc(ctx, tmp, sizeof(uint32_t) * slots);
        keys_out = (uint32_t*)dev_alloc(ctx, tmp, sizeof(uint32_t) * slots);
        vals_out = (uint32_t*)dev_alloc(ctx, tmp, sizeof(uint32_t) * slots);
        if (!A.grid_key || !A.grid_val || !keys_out || !vals_out) return fail(S2_ERR_OOM, "vertex sort allocation failed");
        cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, A.grid_key, keys_out, A.grid_val, vals_out, (int)slots, 0,
                                        lvc ? 1 : (int)grid_bits + 1, s);
        sort_tmp = dev_alloc(ctx, tmp, std::max<size_t>(sort_bytes, 16));
        if (!sort_tmp) return fail(S2_ERR_OOM, "vertex sort scratch allocation failed");
        A.grid_slot = vals_out;
        A.lvc_list = vals_out;
        A.lvc_total = lvc_count;
    }
    // outputs: device pointers directly, host outputs through device scratch
    const bool host = out_on_host != 0;
    float4* rad = nullptr;
    auto dev_out = [&](void* user, size_t bytes) -> void* {
        if (!out || !user) return nullptr;
        return host ? dev_alloc(ctx, tmp, bytes) : user;
    };
    rad = (float4*)dev_out(out ? out->radiance : nullptr, sizeof(float4) * pixels);
    A.aov_albedo = (float4*)dev_out(out ? out->albedo : nullptr, sizeof(float4) * pixels);
    A.aov_vis = (uint2*)dev_out(out ? out->visibility : nullptr, sizeof(uint2) * pixels);
    A.aov_depth = (float4*)dev_out(out ? out->depth : nullptr, sizeof(float4) * pixels);
    A.aov_prev_uv = (float2*)dev_out(out ? out->prev_uv : nullptr, sizeof(float2) * pixels);
    A.aov_ids = (uint2*)dev_out(out ? out->ids32 : nullptr, sizeof(uint2) * pixels);
    if (A.light_trace_only) {  // no camera paths: the AOVs are cleared to zero
        if (A.aov_albedo) cudaMemsetAsync(A.aov_albedo, 0, 16ull * pixels, s);
        if (A.aov_vis) cudaMemsetAsync(A.aov_vis, 0, 8ull * pixels, s);
        if (A.aov_depth) cudaMemsetAsync(A.aov_depth, 0, 16ull * pixels, s);
        if (A.aov_prev_uv) cudaMemsetAsync(A.aov_prev_uv, 0, 8ull * pixels, s);
        if (A.aov_ids) cudaMemsetAsync(A.aov_ids, 0, 8ull * pixels, s);
    }

    cudaMemsetAsync(A.image_fx, 0, 32ull * pixels, s);
    cudaMemsetAsync(A.counts, 0, 4 * sizeof(unsigned long long), s);
    cudaMemsetAsync(ctx->status_dev, 0, sizeof(int), s);
    cudaEventRecord(ctx->ev0, s);
    const bool lam = (prm->flags & S2_FLAG_LAMBERTIAN) != 0;
    uint64_t launches = 0;
    for (uint32_t it = 0; it < prm->iterations; ++it) {
        A.seed = prm->frame_seed + it;
        A.write_aovs = it == 0 ? 1u : 0u;
        // VCM.cpp:449-469: merge radius schedule, normalisation and the MIS weight factors
        const double vm_it = (double)prm->first_iteration + (double)it;
        double radius = (double)prm->merge_radius_factor * (double)R / std::pow(vm_it + 1.0, 0.5 * (1.0 - (double)prm->merge_radius_alpha));
        radius = std::max(radius, 1e-7);
        const double r2 = radius * radius;
        const double eta = M_PI * r2 * (double)n_light;
        A.merge_radius = (float)radius;
        A.cell_size = (float)(2.0 * radius);
        A.vm_norm = (float)(1.0 / eta);
        A.vm_weight = use_vm ? (float)(eta * eta) : 0.f;
        A.vc_weight = use_vc ? (float)(1.0 / (eta * eta)) : 0.f;
        if (!A.path_trace_only) {
            if (lam) launch_light<true>(A, s); else launch_light<false>(A, s);
            launches += 1;
        }
        if (sort && slots > 0) {
            cudaMemsetAsync(lvc_count, 0, sizeof(unsigned int), s);
            vk::k_vcm_keys<<<std::min<uint32_t>((slots + 255) / 256, 148u * 16u), 256, 0, s>>>(A, lvc_count);
            cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, A.grid_key, keys_out, A.grid_val, vals_out, (int)slots, 0,
                                            lvc ? 1 : (int)grid_bits + 1, s);
            launches += 2;
            if (use_vm) {
                cudaMemsetAsync(A.grid_start, 0, sizeof(uint32_t) << grid_bits, s);
                cudaMemsetAsync(A.grid_end, 0, sizeof(uint32_t) << grid_bits, s);
                vk::k_vcm_ranges<<<std::min<uint32_t>((slots + 255) / 256, 148u * 16u), 256, 0, s>>>(A, keys_out);
                launches += 1;
            }
        }
        if (!A.light_trace_only) {
            DiGrid* cur = nullptr;
            if (di_reuse) {
                cur = &vs->grid[vs->cur];
                const HashGridDev& g = cur->g;
                cudaMemsetAsync(g.checksums, 0, sizeof(uint32_t) * g.cell_count, s);  // GpuHashGrid::clear
                cudaMemsetAsync(g.cell_counters, 0, sizeof(uint32_t) * g.cell_count, s);
                cudaMemsetAsync(g.other, 0, sizeof(uint32_t) * 4, s);
                A.di_cur = g;
                A.di_prev = vs->grid[vs->cur ^ 1].g;
                A.di_prev_valid = vs->prev_valid ? 1u : 0u;
            }
            DiGrid* lcur = nullptr;
            if (lvc_reuse) {
                lcur = &vs->lvc_grid[vs->lvc_cur];
                const HashGridDev& g = lcur->g;
                cudaMemsetAsync(g.checksums, 0, sizeof(uint32_t) * g.cell_count, s);
                cudaMemsetAsync(g.cell_counters, 0, sizeof(uint32_t) * g.cell_count, s);
                cudaMemsetAsync(g.other, 0, sizeof(uint32_t) * 4, s);
                A.lvc_cur = g;
                A.lvc_cur_rec = (vk::LvcRecord*)lcur->wide;
                const DiGrid& prev = vs->lvc_grid[vs->lvc_cur ^ 1];
                A.lvc_prev = prev.g;
                A.lvc_prev_rec = (const vk::LvcRecord*)prev.wide;
                A.lvc_prev_valid = vs->lvc_prev_valid ? 1u : 0u;
            }
            if (lam) launch_camera<true>(A, s); else launch_camera<false>(A, s);
            launches += 1;
            if (cur) {  // this iteration's reservoirs become the next one's previous grid
                launches += build_di_grid(*cur, s);
                vs->cur ^= 1u;
                vs->prev_valid = true;
            }
            if (lcur) {
                launches += build_di_grid(*lcur, s);
                vs->lvc_cur ^= 1u;
                vs->lvc_prev_valid = true;
            }
        }
    }
    if (rad) {
        vk::k_resolve_fx<<<(pixels + 255) / 256, 256, 0, s>>>(A.image_fx, 0, pixels,
                                                              exp2f(prm->exposure) / (float)prm->iterations, rad);
        launches += 1;
    }
    cudaEventRecord(ctx->ev1, s);
    int rc = check_cuda(ctx, cudaGetLastError(), "VCM render launch");
    if (rc != S2_OK) { cudaStreamSynchronize(s); free_bufs(tmp); return rc; }
    if (host && out) {
        if (out->radiance) cudaMemcpyAsync(out->radiance, rad, sizeof(float4) * pixels, cudaMemcpyDeviceToHost, s);
        if (out->albedo) cudaMemcpyAsync(out->albedo, A.aov_albedo, sizeof(float4) * pixels, cudaMemcpyDeviceToHost, s);
        if (out->visibility) cudaMemcpyAsync(out->visibility, A.aov_vis, sizeof(uint2) * pixels, cudaMemcpyDeviceToHost, s);
        if (out->depth) cudaMemcpyAsync(out->depth, A.aov_depth, sizeof(float4) * pixels, cudaMemcpyDeviceToHost, s);
        if (out->prev_uv) cudaMemcpyAsync(out->prev_uv, A.aov_prev_uv, sizeof(float2) * pixels, cudaMemcpyDeviceToHost, s);
        if (out->ids32) cudaMemcpyAsync(out->ids32, A.aov_ids, sizeof(uint2) * pixels, cudaMemcpyDeviceToHost, s);
    }
    unsigned long long counts[4] = {0, 0, 0, 0};
    int status = 0;
    cudaMemcpyAsync(counts, A.counts, sizeof(counts), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&status, ctx->status_dev, sizeof(int), cudaMemcpyDeviceToHost, s);
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "VCM render");
    float ms = 0.f;
    if (rc == S2_OK) cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    free_bufs(tmp);
    if (rc != S2_OK) return rc;
    if (status) return set_error(ctx, S2_ERR_DEVICE, "traversal stack overflow during VCM render");
    if (stats_out) {
        std::memset(stats_out, 0, sizeof(*stats_out));
        stats_out->extension_rays = counts[0];
        stats_out->shadow_rays = counts[1];
        stats_out->nan_count = counts[2];
        stats_out->paths = (uint64_t)pixels * prm->iterations;
        stats_out->gpu_ms = ms;
        stats_out->kernel_launches = launches;
    }
    return S2_OK;
}
