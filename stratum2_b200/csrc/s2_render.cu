// s2_render: host orchestration of the wavefront path tracer (replaces TestRenderer::render,
// src/App/TestRenderer.cpp:284-763: per-frame dispatch of Render, RenderIteration x (maxDepth-1),
// ProcessShadowRays and ProcessAtomicOutput).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include <cub/device/device_radix_sort.cuh>

#include "s2_context.h"
#include "s2_shade_kernel.cuh"
#include "s2_light_trace.cuh"

namespace s2 {

// Paths per wave (and batched queue capacity) when neither the call nor the tuning sets one: 2^26
// paths hold about 14 GB of queues, hits and shadow rays.
constexpr uint32_t kDefaultWavePaths = 1u << 26;

struct RenderState {
    uint32_t capacity = 0;      // paths per wave
    uint32_t pixels = 0, width = 0, height = 0;
    std::vector<DevBuf> bufs;   // queues, hits, shadow queue, accumulators
    std::vector<DevBuf> pixel_bufs;
    PathQueue q[2]{};
    float4* hits = nullptr;
    float4 *sh_o = nullptr, *sh_d = nullptr, *sh_c = nullptr;
    float4* accum = nullptr;
    float4* total = nullptr;        // per-pixel sum over all samples so far
    float4* out_radiance = nullptr; // device radiance AOV when the caller's buffers are on the host
    float4* aov_albedo = nullptr;
    uint2* aov_vis = nullptr;
    float4* aov_depth = nullptr;
    float2* aov_prev_uv = nullptr;
    uint2* aov_ids = nullptr;
    uint32_t* hint_tri = nullptr;  // per pixel: the centre ray's triangle (k_pixel_hint)
    uint32_t* counters = nullptr;
    unsigned long long* stats = nullptr;
    uint64_t accumulated_spp = 0;
    int ext_blocks = 0, occ_blocks = 0, shade_blocks = 0;
    int shade_blocks_rc = 0;   // ReSTIR / radiance-cache shade variants (more registers)
    int sort_blocks = 0;
    std::vector<cudaEvent_t> events;  // reusable start/stop pairs for S2_FLAG_PROFILE_KERNELS
    // host outputs: the first-hit AOVs are copied on a side stream while the later bounces render
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t aov_ready = nullptr, copies_done = nullptr;
    // ReSTIR DI reuse: the grid appended to by this call and the previous call's grid
    struct Grid {
        std::vector<DevBuf> bufs;
        HashGridDev g{};
        // build: sort keys in and out, record indices in, CUB temporary storage
        unsigned long long *keys_in = nullptr, *keys_out = nullptr;
        uint32_t* vals_in = nullptr;
        void* sort_tmp = nullptr;
        size_t sort_bytes = 0;
        int end_bit = 64;
    } grid[2];
    uint32_t grid_cur = 0;
    bool grid_prev_valid = false;
    // light tracing: fixed-point per-pixel totals of the camera connections
    std::vector<DevBuf> lt_bufs;
    unsigned long long* lt_fx = nullptr;
    uint32_t lt_pixels = 0;
    // screen-space ReSTIR DI reuse: per-pixel reservoirs of this call and of the previous one
    std::vector<DevBuf> ss_bufs;
    ReservoirRecord* ss[2] = {nullptr, nullptr};
    uint32_t ss_cur = 0, ss_pixels = 0, ss_width = 0;
    bool ss_prev_valid = false;
    // material-key sort buffers (S2Tuning::shade_order)
    std::vector<DevBuf> sort_bufs;
    uint32_t* sort_keys = nullptr;
    uint32_t* sort_perm = nullptr;
    uint32_t* sort_hist = nullptr;
    uint32_t sort_cap = 0;
    // radiance cache queues: terminal-vertex queries and training vertices
    std::vector<DevBuf> cache_bufs;
    float4 *cq_pos = nullptr, *cq_thr = nullptr, *tr_pos = nullptr, *tr_thr = nullptr, *tr_rad = nullptr;
    uint32_t cq_cap = 0, tr_cap = 0;
};

void destroy_batch_state(S2Context* ctx);

void destroy_render_state(S2Context* ctx) {
    destroy_batch_state(ctx);
    if (!ctx->render) return;
    for (cudaEvent_t e : ctx->render->events) cudaEventDestroy(e);
    if (ctx->render->copy_stream) cudaStreamDestroy(ctx->render->copy_stream);
    if (ctx->render->aov_ready) cudaEventDestroy(ctx->render->aov_ready);
    if (ctx->render->copies_done) cudaEventDestroy(ctx->render->copies_done);
    for (auto& g : ctx->render->grid) free_bufs(g.bufs);
    free_bufs(ctx->render->cache_bufs);
    free_bufs(ctx->render->sort_bufs);
    free_bufs(ctx->render->ss_bufs);
    free_bufs(ctx->render->lt_bufs);
    free_bufs(ctx->render->bufs);
    free_bufs(ctx->render->pixel_bufs);
    delete ctx->render;
    ctx->render = nullptr;
}

namespace {

template <typename T>
T* alloc(S2Context* ctx, std::vector<DevBuf>& owner, size_t n) {
    return (T*)dev_alloc(ctx, owner, n * sizeof(T));
}

int ensure_state(S2Context* ctx, uint32_t width, uint32_t height, uint32_t capacity) {
    RenderState* st = ctx->render;
    if (!st) {
        st = ctx->render = new (std::nothrow) RenderState();
        if (!st) return set_error(ctx, S2_ERR_OOM, "render state allocation failed");
        cudaDeviceProp prop;
        cudaGetDeviceProperties(&prop, ctx->device);
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_extend<false>, kTravBlock, 0);
        st->ext_blocks = std::max(1, b) * prop.multiProcessorCount;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_occlude<false>, kTravBlock, 0);
        st->occ_blocks = std::max(1, b) * prop.multiProcessorCount;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_shade<false, false>, 128, 0);
        st->shade_blocks = std::max(1, b) * prop.multiProcessorCount;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_shade<false, true, true>, 128, 0);
        st->shade_blocks_rc = std::max(1, b) * prop.multiProcessorCount;
        st->sort_blocks = 8 * prop.multiProcessorCount;
    }
    const uint32_t pixels = width * height;
    if (st->pixels != pixels || st->width != width) {
        free_bufs(st->pixel_bufs);
        st->total = alloc<float4>(ctx, st->pixel_bufs, pixels);
        st->out_radiance = alloc<float4>(ctx, st->pixel_bufs, pixels);
        st->aov_albedo = alloc<float4>(ctx, st->pixel_bufs, pixels);
        st->aov_vis = alloc<uint2>(ctx, st->pixel_bufs, pixels);
        st->aov_depth = alloc<float4>(ctx, st->pixel_bufs, pixels);
        st->aov_prev_uv = alloc<float2>(ctx, st->pixel_bufs, pixels);
        st->aov_ids = alloc<uint2>(ctx, st->pixel_bufs, pixels);
        st->hint_tri = alloc<uint32_t>(ctx, st->pixel_bufs, pixels);
        st->counters = alloc<uint32_t>(ctx, st->pixel_bufs, C_COUNT);
        st->stats = alloc<unsigned long long>(ctx, st->pixel_bufs, S_COUNT);
        if (!st->total || !st->out_radiance || !st->aov_albedo || !st->aov_vis || !st->aov_depth || !st->aov_prev_uv ||
            !st->aov_ids || !st->hint_tri || !st->counters || !st->stats) {
            free_bufs(st->pixel_bufs);
            st->pixels = 0;
            return S2_ERR_OOM;
        }
        cudaMemsetAsync(st->total, 0, sizeof(float4) * pixels, ctx->stream);
        st->pixels = pixels; st->width = width; st->height = height;
        st->accumulated_spp = 0;
    }
    if (st->capacity < capacity) {
        free_bufs(st->bufs);
        st->capacity = 0;
        for (int k = 0; k < 2; ++k) {
            st->q[k].s0 = alloc<float4>(ctx, st->bufs, capacity);
            st->q[k].s1 = alloc<float4>(ctx, st->bufs, capacity);
            st->q[k].s2 = alloc<float4>(ctx, st->bufs, capacity);
            st->q[k].s3 = alloc<uint4>(ctx, st->bufs, capacity);
        }
        st->hits = alloc<float4>(ctx, st->bufs, capacity);
        st->sh_o = alloc<float4>(ctx, st->bufs, capacity);
        st->sh_d = alloc<float4>(ctx, st->bufs, capacity);
        st->sh_c = alloc<float4>(ctx, st->bufs, capacity);
        st->accum = alloc<float4>(ctx, st->bufs, capacity);
        for (auto& b : st->bufs) if (!b.ptr) return S2_ERR_OOM;
        if (st->bufs.size() != 13) { free_bufs(st->bufs); return S2_ERR_OOM; }
        cudaMemsetAsync(st->accum, 0, sizeof(float4) * capacity, ctx->stream);
        st->capacity = capacity;
    }
    return S2_OK;
}

// Inverse of a row-major 3x4 affine transform (the world-to-camera matrix of a view), in double.
void invert_affine(const float* m, float* out) {
    double a[3][3], t[3];
    for (int r = 0; r < 3; ++r) { for (int c = 0; c < 3; ++c) a[r][c] = m[4 * r + c]; t[r] = m[4 * r + 3]; }
    const double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                       a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    const double id = det != 0.0 ? 1.0 / det : 0.0;
    double inv[3][3];
    inv[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) * id;
    inv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) * id;
    inv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) * id;
    inv[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) * id;
    inv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) * id;
    inv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) * id;
    inv[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) * id;
    inv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) * id;
    inv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) * id;
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) out[4 * r + c] = (float)inv[r][c];
        out[4 * r + 3] = (float)-(inv[r][0] * t[0] + inv[r][1] * t[1] + inv[r][2] * t[2]);
    }
}

// Counting sort of the live queue by material key into P.sort_perm (histogram, scan, scatter).
void launch_sort(const PTParams& P, uint32_t parity, uint32_t blocks, cudaStream_t s) {
    cudaMemsetAsync(P.sort_hist, 0, sizeof(uint32_t) * kSortBuckets, s);
    k_sort_hist<<<blocks, 256, 0, s>>>(P, parity);
    k_sort_scan<<<1, 1024, 0, s>>>(P);
    k_sort_scatter<<<blocks, 256, 0, s>>>(P, parity);
}

// Material-sort buffers for `cap` paths.
int ensure_sort(S2Context* ctx, RenderState* st, uint32_t cap) {
    if (st->sort_cap >= cap) return S2_OK;
    free_bufs(st->sort_bufs);
    st->sort_cap = 0;
    st->sort_keys = alloc<uint32_t>(ctx, st->sort_bufs, cap);
    st->sort_perm = alloc<uint32_t>(ctx, st->sort_bufs, cap);
    st->sort_hist = alloc<uint32_t>(ctx, st->sort_bufs, kSortBuckets);
    if (!st->sort_keys || !st->sort_perm || !st->sort_hist) { free_bufs(st->sort_bufs); return S2_ERR_OOM; }
    st->sort_cap = cap;
    return S2_OK;
}

// Radiance-cache queues: `cq` terminal-vertex queries and `tr` training vertices.
int ensure_cache_queues(S2Context* ctx, RenderState* st, uint32_t cq, uint32_t tr) {
    if (st->cq_cap >= cq && st->tr_cap >= tr) return S2_OK;
    free_bufs(st->cache_bufs);
    st->cq_cap = st->tr_cap = 0;
    cq = std::max(cq, st->cq_cap);
    st->cq_pos = alloc<float4>(ctx, st->cache_bufs, cq);
    st->cq_thr = alloc<float4>(ctx, st->cache_bufs, cq);
    st->tr_pos = alloc<float4>(ctx, st->cache_bufs, tr);
    st->tr_thr = alloc<float4>(ctx, st->cache_bufs, tr);
    st->tr_rad = alloc<float4>(ctx, st->cache_bufs, tr);
    for (auto& b : st->cache_bufs) if (!b.ptr) { free_bufs(st->cache_bufs); return S2_ERR_OOM; }
    if (st->cache_bufs.size() != 5) { free_bufs(st->cache_bufs); return S2_ERR_OOM; }
    st->cq_cap = cq;
    st->tr_cap = tr;
    return S2_OK;
}

// Builds a grid after its appends (cell offsets by a scan, records sorted by cell and content);
// returns the kernel launches issued.
uint32_t build_grid(S2Context* ctx, RenderState::Grid& G, cudaStream_t s) {
    const HashGridDev& g = G.g;
    k_hg_scan<<<1, kHgScanThreads, 0, s>>>(g);
    k_hg_keys<<<(g.max_size + 255) / 256, 256, 0, s>>>(g, G.keys_in, G.vals_in);
    size_t bytes = G.sort_bytes;
    cub::DeviceRadixSort::SortPairs(G.sort_tmp, bytes, G.keys_in, G.keys_out, G.vals_in, g.data_indices, (int)g.max_size, 0,
                                    G.end_bit, s);
    (void)ctx;
    return 3;
}

// (Re)allocates one hash grid for `cells` cells and `size` records (GpuHashGrid::init,
// src/App/GpuHashGrid.cpp:17-69).
int ensure_grid(S2Context* ctx, RenderState::Grid& G, uint32_t cells, uint32_t size) {
    if (G.g.checksums && G.g.cell_count == cells && G.g.max_size >= size) return S2_OK;
    free_bufs(G.bufs);
    G.g = HashGridDev{};
    HashGridDev g{};
    g.checksums = alloc<uint32_t>(ctx, G.bufs, cells);
    g.cell_counters = alloc<uint32_t>(ctx, G.bufs, cells);
    g.other = alloc<uint32_t>(ctx, G.bufs, 4);
    g.append_indices = alloc<uint2>(ctx, G.bufs, size);
    g.data = alloc<ReservoirRecord>(ctx, G.bufs, size);
    g.indices = alloc<uint32_t>(ctx, G.bufs, cells);
    g.data_indices = alloc<uint32_t>(ctx, G.bufs, size);
    G.keys_in = alloc<unsigned long long>(ctx, G.bufs, size);
    G.keys_out = alloc<unsigned long long>(ctx, G.bufs, size);
    G.vals_in = alloc<uint32_t>(ctx, G.bufs, size);
    // keys: cell (bits 32 and up) above a 32-bit content hash; unused slots take cell `cells`, one
    // past the last, so they sort last; the sort reads 32 + ceil(log2(cells + 1)) bits
    int cell_bits = 1;
    while (cell_bits < 32 && (1ull << cell_bits) <= cells) ++cell_bits;
    G.end_bit = 32 + cell_bits;
    G.sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, G.sort_bytes, G.keys_in, G.keys_out, G.vals_in, g.data_indices, (int)size, 0,
                                    G.end_bit, ctx->stream);
    G.sort_tmp = dev_alloc(ctx, G.bufs, std::max<size_t>(G.sort_bytes, 16));
    for (auto& b : G.bufs) if (!b.ptr) { free_bufs(G.bufs); return S2_ERR_OOM; }
    if (G.bufs.size() != 11) { free_bufs(G.bufs); return S2_ERR_OOM; }
    g.cell_count = cells;
    g.max_size = size;
    G.g = g;
    return S2_OK;
}

template <bool L, bool R>
void launch_shade(const PTParams& P, uint32_t parity, const RenderState* st, cudaStream_t s) {
    if (P.cache_on) k_shade<L, R, true><<<st->shade_blocks_rc, 128, 0, s>>>(P, parity);
    else k_shade<L, R><<<R ? st->shade_blocks_rc : st->shade_blocks, 128, 0, s>>>(P, parity);
}

// One baked shading record per BVH triangle (make_shading_rec): triangles of mesh instances whose
// vertex data has neither texture coordinates nor normals get the per-triangle terms of
// shading_terms, the function the gathered path runs; the others are marked invalid and keep the
// gather chain.
__global__ void k_bake_shading(const __grid_constant__ DevScene s, float4* __restrict__ recs) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.tri_count) return;
    float4* out = recs + 4 * (size_t)i;
    out[3] = make_float4(0.f, 0.f, 0.f, 0.f);  // invalid unless baked below
    const uint32_t inst = __float_as_uint(s.tris[3 * (size_t)i].w), prim = __float_as_uint(s.tris[3 * (size_t)i + 1].w);
    const uint2 id = s.instances[inst];
    if ((id.x & 0xfu) != S2_INSTANCE_TYPE_MESH) return;
    const VInfo vi = load_vinfo(s, id.y & 0xffffu);
    if (vi_texcoord_buffer(vi) < s.vbuf_count || vi_normal_buffer(vi) < s.vbuf_count) return;
    SD sd;
    float3 v0, e1, e2;
    shading_terms(s, inst, prim, 0.f, 0.f, false, sd, v0, e1, e2);
    out[0] = make_float4(v0.x, v0.y, v0.z, __uint_as_float(sd.mat));
    out[1] = make_float4(e1.x, e1.y, e1.z, sd.area);
    out[2] = make_float4(e2.x, e2.y, e2.z, __uint_as_float(sd.ng));
    out[3] = make_float4(__uint_as_float(sd.tg), __uint_as_float(kShadeRecValid), 0.f, 0.f);
}

}  // namespace

// Builds the baked shading records of the current BVH (called by s2_build_bvh).
int bake_shading_records(S2Context* ctx, std::vector<DevBuf>& owner) {
    ctx->scene.shade_recs = nullptr;
    const uint32_t n = ctx->scene.tri_count;
    if (n == 0) return S2_OK;
    float4* recs = (float4*)dev_alloc(ctx, owner, sizeof(float4) * 4 * (size_t)n);
    if (!recs) return set_error(ctx, S2_ERR_OOM, "shading record allocation failed");
    k_bake_shading<<<(n + 255) / 256, 256, 0, ctx->stream>>>(ctx->scene, recs);
    const int rc = check_cuda(ctx, cudaGetLastError(), "shading record bake");
    if (rc == S2_OK) ctx->scene.shade_recs = recs;
    return rc;
}
}  // namespace s2

using namespace s2;

extern "C" void s2_default_render_params(S2RenderParams* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->min_path_length = 0;
    p->max_path_length = 5;         // mMaxDepth (TestRenderer.cpp:38)
    p->exposure = 0.f;
    p->spp = 1;
    p->environment_sample_probability = 0.9f;  // TestRenderer.cpp:41
    p->restir_candidates = 32;      // TestRenderer.cpp:42
    p->restir_max_m = 3.f;          // TestRenderer.cpp:43
    p->restir_grid_cells = 100000;  // TestRenderer.cpp:52
    p->restir_grid_cell_size = 0.5f;
}

extern "C" int s2_render(S2Context* ctx, const S2View* view, const S2RenderParams* prm, const S2Aovs* out, int out_on_host,
                         S2RenderStats* stats_out) {
    if (!ctx) return S2_ERR_INVALID;
    if (!view || !prm) return set_error(ctx, S2_ERR_INVALID, "view and params are required");
    if (!ctx->has_bvh) return set_error(ctx, S2_ERR_NO_SCENE, "s2_render before s2_scene_upload + s2_build_bvh");
    const int W = view->image_max[0] - view->image_min[0], H = view->image_max[1] - view->image_min[1];
    if (W <= 0 || H <= 0 || (int64_t)W * H > (1ll << 28)) return set_error(ctx, S2_ERR_INVALID, "invalid view extent");
    if (prm->spp == 0) return set_error(ctx, S2_ERR_INVALID, "spp must be >= 1");
    if (prm->max_path_length > 255) return set_error(ctx, S2_ERR_INVALID, "max_path_length must be <= 255");
    if ((prm->flags & S2_FLAG_RESTIR_DI) && (prm->restir_candidates == 0 || prm->restir_candidates > 1024))
        return set_error(ctx, S2_ERR_INVALID, "restir_candidates must be in 1..1024");
    const bool reuse = (prm->flags & S2_FLAG_RESTIR_DI) && (prm->flags & S2_FLAG_RESTIR_REUSE);
    const bool screen = (prm->flags & S2_FLAG_RESTIR_DI) && (prm->flags & S2_FLAG_RESTIR_SCREEN);
    const bool light_trace = (prm->flags & S2_FLAG_LIGHT_TRACE) != 0;
    if (light_trace) {
        if (prm->flags & (S2_FLAG_RESTIR_DI | S2_FLAG_RESTIR_REUSE | S2_FLAG_RESTIR_SCREEN | S2_FLAG_RADIANCE_CACHE))
            return set_error(ctx, S2_ERR_UNSUPPORTED, "light tracing takes no ReSTIR or radiance-cache flags");
        if (!(prm->light_subpaths >= 0.f) || !std::isfinite(prm->light_subpaths))
            return set_error(ctx, S2_ERR_INVALID, "light_subpaths must be finite and >= 0");
    }
    if ((prm->flags & S2_FLAG_RESTIR_REUSE) && (prm->flags & S2_FLAG_RESTIR_SCREEN))
        return set_error(ctx, S2_ERR_INVALID, "S2_FLAG_RESTIR_REUSE and S2_FLAG_RESTIR_SCREEN are exclusive");
    if (screen && (prm->restir_spatial > 32 || !(prm->restir_spatial_radius >= 0.f) || !std::isfinite(prm->restir_spatial_radius) ||
                   !(prm->restir_max_m > 0.f)))
        return set_error(ctx, S2_ERR_INVALID, "invalid screen-space ReSTIR parameters (restir_spatial <= 32, "
                                              "restir_spatial_radius >= 0, restir_max_m > 0)");
    const bool cache = (prm->flags & S2_FLAG_RADIANCE_CACHE) != 0;
    if (cache && !ctx->cache) return set_error(ctx, S2_ERR_INVALID, "S2_FLAG_RADIANCE_CACHE needs s2_cache_init");
    if (reuse && (prm->restir_grid_cells > (1u << 26) || prm->restir_grid_cell_size < 0.f ||
                  !std::isfinite(prm->restir_grid_cell_size) || !(prm->restir_grid_pixel_radius >= 0.f) ||
                  !std::isfinite(prm->restir_grid_pixel_radius) || !(prm->restir_max_m > 0.f)))
        return set_error(ctx, S2_ERR_INVALID, "invalid ReSTIR hash-grid parameters");
    cudaSetDevice(ctx->device);
    const uint32_t pixels = (uint32_t)W * (uint32_t)H;
    uint64_t target = prm->wave_paths ? prm->wave_paths : (ctx->tuning.wave_paths ? ctx->tuning.wave_paths : kDefaultWavePaths);
    uint32_t slots = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(prm->spp, target / pixels));
    // light tracing: one queue of max(1, pixels x light_subpaths) light subpaths per sample pass
    const uint32_t lt_paths = (uint32_t)std::max(1.0, std::min(4294967040.0, (double)pixels *
                                                 (prm->light_subpaths > 0.f ? (double)prm->light_subpaths : 1.0)));
    const uint32_t capacity = light_trace ? lt_paths : slots * pixels;
    int rc = ensure_state(ctx, (uint32_t)W, (uint32_t)H, capacity);
    if (rc != S2_OK) return rc;
    RenderState* st = ctx->render;
    cudaStream_t s = ctx->stream;

    PTParams P;
    std::memset(&P, 0, sizeof(P));
    P.scene = ctx->scene;
    if (ctx->tuning.shade_records == S2_SHADE_RECORDS_OFF) P.scene.shade_recs = nullptr;
    P.scene.light_power_pick = (prm->flags & S2_FLAG_LIGHT_POWER_PICK) ? 1u : 0u;
    P.scene.env_fp_on = (prm->flags & S2_FLAG_ENV_FOOTPRINT_PDF) ? 1u : 0u;
    P.scene.env_sample_prob = prm->environment_sample_probability > 0.f ? prm->environment_sample_probability : 0.9f;
    std::memcpy(P.proj, view->projection, sizeof(P.proj));
    P.imin[0] = view->image_min[0]; P.imin[1] = view->image_min[1];
    P.imax[0] = view->image_max[0]; P.imax[1] = view->image_max[1];
    std::memcpy(P.cam, view->camera_to_world, sizeof(P.cam));
    std::memcpy(P.prev_inv, view->prev_world_to_camera, sizeof(P.prev_inv));
    P.width = (uint32_t)W; P.height = (uint32_t)H; P.pixels = pixels;
    P.min_len = prm->min_path_length;
    P.max_len = prm->max_path_length;
    P.flags = prm->flags;
    P.frame_seed = prm->frame_seed;
    P.restir_m = prm->restir_candidates ? prm->restir_candidates : 32;
    P.exposure = prm->exposure;
    P.trav.tris_per_step = ctx->tuning.trav_tris_per_step;
    P.trav.vote8 = ctx->tuning.trav_vote8;
    P.refill_min = ctx->tuning.refill_min;
    const bool sort = ctx->tuning.shade_order == S2_SHADE_ORDER_MATERIAL;
    const bool ray_sort = ctx->tuning.trace_order == S2_TRACE_ORDER_COHERENT;
    if (sort || ray_sort) {
        rc = ensure_sort(ctx, st, capacity);
        if (rc != S2_OK) return set_error(ctx, rc, "sort buffer allocation failed");
        P.sort_on = sort; P.ray_sort_on = ray_sort;
        P.sort_keys = st->sort_keys; P.sort_perm = st->sort_perm; P.sort_hist = st->sort_hist;
    }
    P.q[0] = st->q[0]; P.q[1] = st->q[1];
    P.hits = st->hits; P.sh_o = st->sh_o; P.sh_d = st->sh_d; P.sh_c = st->sh_c;
    P.accum = st->accum;
    P.counters = st->counters;
    P.stats = st->stats;
    P.status = ctx->status_dev;
    const bool host = out_on_host != 0;
    auto pick = [&](void* user, void* internal) -> void* { return !out ? nullptr : (user ? (host ? internal : user) : nullptr); };
    P.aov_albedo = (float4*)pick(out ? out->albedo : nullptr, st->aov_albedo);
    P.aov_vis = (uint2*)pick(out ? out->visibility : nullptr, st->aov_vis);
    P.aov_depth = (float4*)pick(out ? out->depth : nullptr, st->aov_depth);
    P.aov_prev_uv = (float2*)pick(out ? out->prev_uv : nullptr, st->aov_prev_uv);
    P.aov_ids = (uint2*)pick(out ? out->ids32 : nullptr, st->aov_ids);

    if (reuse) {
        // TestRenderer.cpp:472-493 and :595-628: this call appends to one grid while reading the
        // previous call's; the grid holds pixels x min(2, maxDepth-1) records per sample pass
        // (appends beyond that are dropped, as in HashGrid::Append).
        const uint32_t cells = prm->restir_grid_cells ? prm->restir_grid_cells : 100000u;
        const uint64_t per_pass = (uint64_t)pixels * std::max(1u, std::min(2u, prm->max_path_length ? prm->max_path_length - 1 : 1u));
        const uint32_t size = (uint32_t)std::min<uint64_t>(per_pass * prm->spp, 1u << 24);
        RenderState::Grid& cur = st->grid[st->grid_cur];
        RenderState::Grid& prev = st->grid[st->grid_cur ^ 1];
        rc = ensure_grid(ctx, cur, cells, size);
        if (rc != S2_OK) return set_error(ctx, rc, "hash grid allocation failed");
        HashGridDev& g = cur.g;
        g.min_cell_size = prm->restir_grid_cell_size > 0.f ? prm->restir_grid_cell_size : 0.5f;
        g.cell_pixel_radius = prm->restir_grid_pixel_radius;
        g.camera_position = make_float3(view->camera_to_world[3], view->camera_to_world[7], view->camera_to_world[11]);
        // GpuHashGrid.cpp:34: tan(radius * vfov * max(1/h, h/w^2))
        g.distance_scale = tanf(g.cell_pixel_radius * view->projection[7] *
                                std::max(1.f / (float)H, (float)H / ((float)W * (float)W)));
        cudaMemsetAsync(g.checksums, 0, sizeof(uint32_t) * cells, s);       // GpuHashGrid::clear
        cudaMemsetAsync(g.cell_counters, 0, sizeof(uint32_t) * cells, s);
        cudaMemsetAsync(g.other, 0, sizeof(uint32_t) * 4, s);
        P.grid_cur = g;
        P.grid_prev = prev.g;
        P.prev_valid = st->grid_prev_valid && prev.g.checksums ? 1u : 0u;
        P.reuse = 1;
        P.max_m = prm->restir_max_m;
    } else {
        st->grid_prev_valid = false;  // TestRenderer.cpp:495-498 drops the grids when reuse is off
    }
    if (screen) {
        if (st->ss_pixels != pixels || st->ss_width != (uint32_t)W) {
            free_bufs(st->ss_bufs);
            st->ss_pixels = 0;
            st->ss_prev_valid = false;
            st->ss[0] = alloc<ReservoirRecord>(ctx, st->ss_bufs, pixels);
            st->ss[1] = alloc<ReservoirRecord>(ctx, st->ss_bufs, pixels);
            if (!st->ss[0] || !st->ss[1]) { free_bufs(st->ss_bufs); return set_error(ctx, S2_ERR_OOM, "reservoir buffer allocation failed"); }
            st->ss_pixels = pixels;
            st->ss_width = (uint32_t)W;
        }
        ReservoirRecord* cur = st->ss[st->ss_cur];
        cudaMemsetAsync(cur, 0, sizeof(ReservoirRecord) * pixels, s);  // pixels without a primary vertex: W = 0
        P.ss_on = 1;
        P.ss_cur = cur;
        P.ss_prev = st->ss[st->ss_cur ^ 1u];
        P.ss_prev_valid = st->ss_prev_valid ? 1u : 0u;
        P.ss_spatial = prm->restir_spatial ? prm->restir_spatial : 5u;
        P.ss_radius = prm->restir_spatial_radius > 0.f ? prm->restir_spatial_radius : 30.f;
        P.max_m = prm->restir_max_m;
    } else {
        st->ss_prev_valid = false;
    }
    const uint32_t cache_len = (prm->cache_bounces ? prm->cache_bounces : 2u) + 1u;
    const uint32_t train_paths = prm->cache_train_paths ? prm->cache_train_paths : 65536u;
    if (cache) {
        const uint64_t tr_cap64 = std::min<uint64_t>((uint64_t)train_paths * std::max(1u, prm->max_path_length), 1u << 26);
        rc = ensure_cache_queues(ctx, st, capacity, (uint32_t)tr_cap64);
        if (rc != S2_OK) return set_error(ctx, rc, "radiance cache queue allocation failed");
        P.cache_on = 1;
        P.cache_len = cache_len;
        P.cache_rough = std::min(1.f, std::max(0.f, prm->cache_min_roughness));
        P.cq_pos = st->cq_pos; P.cq_thr = st->cq_thr; P.cq_cap = st->cq_cap;
        P.tr_pos = st->tr_pos; P.tr_thr = st->tr_thr; P.tr_rad = st->tr_rad; P.tr_cap = st->tr_cap;
    }
    if (!(prm->flags & S2_FLAG_ACCUMULATE)) {
        cudaMemsetAsync(st->total, 0, sizeof(float4) * pixels, s);
        st->accumulated_spp = 0;
    }
    if (light_trace) {
        if (st->lt_pixels != pixels) {
            free_bufs(st->lt_bufs);
            st->lt_pixels = 0;
            st->lt_fx = (unsigned long long*)dev_alloc(ctx, st->lt_bufs, 32ull * pixels);
            if (!st->lt_fx) return set_error(ctx, S2_ERR_OOM, "light-tracing accumulator allocation failed");
            st->lt_pixels = pixels;
            cudaMemsetAsync(st->lt_fx, 0, 32ull * pixels, s);
        }
        if (!(prm->flags & S2_FLAG_ACCUMULATE)) cudaMemsetAsync(st->lt_fx, 0, 32ull * pixels, s);
        P.total_fx = st->lt_fx;
        // light tracing has no first camera hit: the other AOVs are cleared to zero
        if (P.aov_albedo) cudaMemsetAsync(P.aov_albedo, 0, 16ull * pixels, s);
        if (P.aov_vis) cudaMemsetAsync(P.aov_vis, 0, 8ull * pixels, s);
        if (P.aov_depth) cudaMemsetAsync(P.aov_depth, 0, 16ull * pixels, s);
        if (P.aov_prev_uv) cudaMemsetAsync(P.aov_prev_uv, 0, 8ull * pixels, s);
        if (P.aov_ids) cudaMemsetAsync(P.aov_ids, 0, 8ull * pixels, s);
        P.aov_albedo = nullptr; P.aov_vis = nullptr; P.aov_depth = nullptr; P.aov_prev_uv = nullptr; P.aov_ids = nullptr;
        P.sort_on = 0; P.ray_sort_on = 0;
        P.lt_paths = lt_paths;
        // ViewData::imagePlaneDist: |image height| / (2 tan(vfov / 2))
        P.lt_image_plane_dist = std::fabs((float)(view->image_max[1] - view->image_min[1])) / (2.f * std::tan(view->projection[7] * 0.5f));
        invert_affine(view->camera_to_world, P.cam_inv);
    }
    cudaMemsetAsync(st->stats, 0, sizeof(unsigned long long) * S_COUNT, s);
    cudaMemsetAsync(ctx->status_dev, 0, sizeof(int), s);
    cudaEventRecord(ctx->ev0, s);
    const bool lam = (prm->flags & S2_FLAG_LAMBERTIAN) != 0, restir = (prm->flags & S2_FLAG_RESTIR_DI) != 0;
    const bool count = (prm->flags & S2_FLAG_COUNT_FETCHES) != 0, prof = (prm->flags & S2_FLAG_PROFILE_KERNELS) != 0;
    uint64_t launches = 0;
    // profiling: an event pair around every extend / shade / occlude launch (kind 0 / 1 / 2)
    std::vector<int> prof_kind;
    auto ev_begin = [&](int kind) {
        if (!prof) return;
        const size_t k = 2 * prof_kind.size();
        while (st->events.size() < k + 2) { cudaEvent_t e; cudaEventCreate(&e); st->events.push_back(e); }
        cudaEventRecord(st->events[k], s);
        prof_kind.push_back(kind);
    };
    auto ev_end = [&]() { if (prof) cudaEventRecord(st->events[2 * prof_kind.size() - 1], s); };
    // Host outputs: the first-hit AOVs are written by wave 0's first shade only, so their copies can
    // run on a side stream while the later bounces render.  They are issued after every kernel of the
    // call is queued, since a copy to pageable memory holds the host until it completes.
    const bool early_aov = host && out && !light_trace &&
                           (out->albedo || out->visibility || out->depth || out->prev_uv || out->ids32);
    if (early_aov) {
        if (!st->copy_stream) cudaStreamCreateWithFlags(&st->copy_stream, cudaStreamNonBlocking);
        if (!st->aov_ready) cudaEventCreateWithFlags(&st->aov_ready, cudaEventDisableTiming);
        if (!st->copies_done) cudaEventCreateWithFlags(&st->copies_done, cudaEventDisableTiming);
        if (!st->copy_stream || !st->aov_ready || !st->copies_done) return set_error(ctx, S2_ERR_CUDA, "copy stream creation failed");
    }
    for (uint32_t sample = 0; light_trace && sample < prm->spp; ++sample) {
        // one light pass: light subpaths, then per vertex the camera connections and continuation
        cudaMemsetAsync(st->counters, 0, sizeof(uint32_t) * C_COUNT, s);
        k_light_gen<<<std::min<uint32_t>((lt_paths + 255) / 256, 148u * 16u), 256, 0, s>>>(P, sample);
        launches += 1;
        for (uint32_t b = 0; b < prm->max_path_length; ++b) {
            const uint32_t parity = b & 1u;
            k_bounce_setup<<<1, 32, 0, s>>>(P, parity, b == 0);
            ev_begin(0);
            if (count) k_extend<true><<<st->ext_blocks, kTravBlock, 0, s>>>(P, parity);
            else k_extend<false><<<st->ext_blocks, kTravBlock, 0, s>>>(P, parity);
            ev_end();
            ev_begin(1);
            if (lam) k_light_shade<true><<<st->shade_blocks, 128, 0, s>>>(P, parity);
            else k_light_shade<false><<<st->shade_blocks, 128, 0, s>>>(P, parity);
            ev_end();
            ev_begin(2);
            if (count) k_occlude<true><<<st->occ_blocks, kTravBlock, 0, s>>>(P);
            else k_occlude<false><<<st->occ_blocks, kTravBlock, 0, s>>>(P);
            ev_end();
            launches += 4;
        }
        k_wave_finish<<<1, 32, 0, s>>>(P);
        launches += 1;
    }
    // shadow rays of bounce b traced by bounce b + 1's k_trace (S2Tuning::shadow_merge; the cache's
    // terminal contributions must land after the NEE of the same vertex, so not with the cache)
    const bool merge = !cache && ctx->tuning.shadow_merge != S2_SHADOW_MERGE_OFF;
    P.sh_merge = merge ? 1u : 0u;
    // frames of 8 or more samples per pixel: every camera ray first tests the triangle its pixel's
    // centre ray hits (one traversal per pixel, once per call), so it starts with a tight t_max
    const bool hint = !light_trace && prm->spp >= 8;
    if (hint) {
        k_pixel_hint<<<(pixels + kTravBlock - 1) / kTravBlock, kTravBlock, 0, s>>>(P, st->hint_tri);
        launches += 1;
    }
    for (uint32_t done = 0; !light_trace && done < prm->spp; done += slots) {
        P.wave_base_sample = done;
        P.wave_samples = std::min(slots, prm->spp - done);
        const uint32_t n = P.wave_samples * pixels;
        if (cache) P.train_mod = std::max(1u, n / train_paths);
        P.sh_parity = 0;
        k_raygen<<<(n + 255) / 256, 256, 0, s>>>(P);
        for (uint32_t b = 0; b < prm->max_path_length; ++b) {
            const uint32_t parity = b & 1u;
            const uint32_t sh_prev = sh_counter(P);  // the previous bounce's shadow rays
            P.sh_parity = merge ? (b & 1u) : 0u;
            k_bounce_setup<<<1, 32, 0, s>>>(P, parity, b == 0);
            P.ray_sorted = ray_sort && b > 0;  // camera rays come in pixel-tile order
            // camera paths are queued pixel by pixel: with 32 or more samples per pixel in the wave
            // a warp's camera paths share a pixel and nearly always its material, so the material
            // sort starts with the first bounce (with fewer, a warp spans several pixels and the
            // camera bounce is sorted too)
            P.sort_on = sort && (b > 0 || P.wave_samples < 32);
            if (P.ray_sorted) { launch_sort(P, parity, st->sort_blocks, s); launches += 3; }
            ev_begin(0);
            P.hint_tri = hint && b == 0 ? st->hint_tri : nullptr;
            if (merge && b > 0) {
                if (count) k_trace<true><<<st->ext_blocks, kTravBlock, 0, s>>>(P, parity, sh_prev);
                else k_trace<false><<<st->ext_blocks, kTravBlock, 0, s>>>(P, parity, sh_prev);
            } else {
                if (count) k_extend<true><<<st->ext_blocks, kTravBlock, 0, s>>>(P, parity);
                else k_extend<false><<<st->ext_blocks, kTravBlock, 0, s>>>(P, parity);
            }
            P.hint_tri = nullptr;
            ev_end();
            if (P.sort_on) { launch_sort(P, parity, st->sort_blocks, s); launches += 3; }
            ev_begin(1);
            if (lam) { if (restir) launch_shade<true, true>(P, parity, st, s); else launch_shade<true, false>(P, parity, st, s); }
            else { if (restir) launch_shade<false, true>(P, parity, st, s); else launch_shade<false, false>(P, parity, st, s); }
            ev_end();
            if (early_aov && done == 0 && b == 0) cudaEventRecord(st->aov_ready, s);  // first-hit AOVs are final
            if (cache && b + 1 == cache_len) {
                rc = cache_apply_device(ctx, st->cq_pos, st->cq_thr, st->cq_cap, st->counters + C_CACHEQ, st->accum);
                if (rc != S2_OK) return rc;
                launches += 1;
            }
            if (!merge) {
                ev_begin(2);
                if (count) k_occlude<true><<<st->occ_blocks, kTravBlock, 0, s>>>(P);
                else k_occlude<false><<<st->occ_blocks, kTravBlock, 0, s>>>(P);
                ev_end();
                launches += 1;
            }
            launches += 3;
        }
        if (merge) {  // the last bounce's shadow rays
            k_occlude_setup<<<1, 32, 0, s>>>(P);
            ev_begin(2);
            if (count) k_occlude<true><<<st->occ_blocks, kTravBlock, 0, s>>>(P);
            else k_occlude<false><<<st->occ_blocks, kTravBlock, 0, s>>>(P);
            ev_end();
            launches += 2;
        }
        if (cache) {
            // training: per-vertex targets from the finished training paths, one optimiser step
            k_cache_targets<<<std::max(1, st->shade_blocks / 2), 256, 0, s>>>(P);
            rc = cache_backward_device(ctx, st->tr_pos, st->tr_rad, st->tr_cap, st->counters + C_TRAIN);
            if (rc == S2_OK) rc = cache_adam_device(ctx, st->tr_cap, st->counters + C_TRAIN);
            if (rc != S2_OK) return rc;
            launches += 5;
        }
        k_wave_finish<<<1, 32, 0, s>>>(P);
        k_reduce<<<(pixels + 255) / 256, 256, 0, s>>>(P, st->total);
        launches += 3;
    }
    if (reuse) {
        // GpuHashGrid::build (GpuHashGrid.cpp:84-111), then this grid becomes the previous one
        launches += build_grid(ctx, st->grid[st->grid_cur], s);
        st->grid_cur ^= 1u;
        st->grid_prev_valid = true;
    }
    if (screen) {  // this call's reservoirs become the previous ones
        st->ss_cur ^= 1u;
        st->ss_prev_valid = true;
    }
    launches += 1;  // resolve
    st->accumulated_spp += prm->spp;
    float4* rad = (out && out->radiance) ? (host ? st->out_radiance : (float4*)out->radiance) : st->out_radiance;
    if (light_trace)
        k_resolve_fx<<<(pixels + 255) / 256, 256, 0, s>>>(st->lt_fx, 0, pixels,
                                                          (float)(1.0 / (double)st->accumulated_spp) * exp2f(prm->exposure), rad);
    else
        k_resolve<<<(pixels + 255) / 256, 256, 0, s>>>(st->total, pixels, (float)(1.0 / (double)st->accumulated_spp),
                                                       exp2f(prm->exposure), rad);
    cudaEventRecord(ctx->ev1, s);
    rc = check_cuda(ctx, cudaGetLastError(), "render kernel launch");
    if (rc != S2_OK) return rc;
    if (host && out) {
        cudaStream_t as = early_aov ? st->copy_stream : s;
        if (early_aov) cudaStreamWaitEvent(as, st->aov_ready, 0);
        if (out->albedo) cudaMemcpyAsync(out->albedo, st->aov_albedo, sizeof(float4) * pixels, cudaMemcpyDeviceToHost, as);
        if (out->visibility) cudaMemcpyAsync(out->visibility, st->aov_vis, sizeof(uint2) * pixels, cudaMemcpyDeviceToHost, as);
        if (out->depth) cudaMemcpyAsync(out->depth, st->aov_depth, sizeof(float4) * pixels, cudaMemcpyDeviceToHost, as);
        if (out->prev_uv) cudaMemcpyAsync(out->prev_uv, st->aov_prev_uv, sizeof(float2) * pixels, cudaMemcpyDeviceToHost, as);
        if (out->ids32) cudaMemcpyAsync(out->ids32, st->aov_ids, sizeof(uint2) * pixels, cudaMemcpyDeviceToHost, as);
        if (early_aov) {  // the call's stream waits for the side copies, so its synchronisation covers them
            cudaEventRecord(st->copies_done, as);
            cudaStreamWaitEvent(s, st->copies_done, 0);
        }
        if (out->radiance) cudaMemcpyAsync(out->radiance, st->out_radiance, sizeof(float4) * pixels, cudaMemcpyDeviceToHost, s);
    }
    if (stats_out || host) {
        unsigned long long sv[S_COUNT] = {0, 0, 0, 0, 0, 0, 0, 0};
        int status = 0;
        cudaMemcpyAsync(sv, st->stats, sizeof(sv), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&status, ctx->status_dev, sizeof(int), cudaMemcpyDeviceToHost, s);
        rc = check_cuda(ctx, cudaStreamSynchronize(s), "render");
        if (rc != S2_OK) return rc;
        if (status & 4) return set_error(ctx, S2_ERR_TIMEOUT, "tensor-core wait timed out in the radiance cache");
        if (status) return set_error(ctx, S2_ERR_DEVICE, "traversal stack overflow during render");
        if (stats_out) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
            stats_out->extension_rays = sv[S_EXT];
            stats_out->shadow_rays = sv[S_SHADOW];
            stats_out->paths = (uint64_t)pixels * prm->spp;
            stats_out->nan_count = sv[S_NAN];
            stats_out->gpu_ms = ms;
            stats_out->kernel_launches = launches;
            stats_out->extend_node_fetches = sv[S_EXT_NODES];
            stats_out->extend_tri_fetches = sv[S_EXT_TRIS];
            stats_out->shadow_node_fetches = sv[S_SH_NODES];
            stats_out->shadow_tri_fetches = sv[S_SH_TRIS];
            double kms[3] = {0, 0, 0};
            uint32_t kn[3] = {0, 0, 0};
            for (size_t k = 0; k < prof_kind.size(); ++k) {
                float t = 0.f;
                cudaEventElapsedTime(&t, st->events[2 * k], st->events[2 * k + 1]);
                kms[prof_kind[k]] += t;
                kn[prof_kind[k]]++;
            }
            stats_out->extend_ms = kms[0]; stats_out->shade_ms = kms[1]; stats_out->occlude_ms = kms[2];
            stats_out->extend_launches = kn[0]; stats_out->shade_launches = kn[1]; stats_out->occlude_launches = kn[2];
        }
    }
    return S2_OK;
}

// ============================================================================== batched rendering
namespace s2 {
namespace {

struct BatchState {
    uint32_t capacity = 0;
    std::vector<DevBuf> qbufs;     // path queues, hits, shadow queue
    PathQueue q[2]{};
    float4* hits = nullptr;
    float4 *sh_o = nullptr, *sh_d = nullptr, *sh_c = nullptr;
    std::vector<DevBuf> pbufs;     // per-pixel accumulators, view table, staging
    uint64_t pixels = 0;
    std::vector<uint32_t> layout;  // view extents of the current accumulators
    unsigned long long* total_fx = nullptr;
    ViewEntry* views_dev = nullptr;
    uint32_t views_cap = 0;
    unsigned long long* stream_state = nullptr;
    uint32_t* counters = nullptr;
    unsigned long long* stats = nullptr;
    unsigned long long* done_host = nullptr;  // pinned
    float4* stage_rad = nullptr;
    uint64_t accumulated_spp = 0;
    std::vector<DevBuf> tbufs;     // radiance-cache training-path accumulators
    float4* train_accum = nullptr;
    uint32_t train_cap = 0;
};

BatchState* g_batch_for(S2Context* ctx);

}  // namespace
}  // namespace s2

// One BatchState per context, kept beside the wave-mode RenderState.
namespace s2 {
namespace {
struct BatchRegistry {
    std::vector<std::pair<S2Context*, BatchState*>> items;
};
BatchRegistry g_registry;
std::mutex g_registry_mutex;
BatchState* g_batch_for(S2Context* ctx) {
    std::lock_guard<std::mutex> lock(g_registry_mutex);
    for (auto& it : g_registry.items) if (it.first == ctx) return it.second;
    BatchState* b = new (std::nothrow) BatchState();
    if (b) g_registry.items.push_back({ctx, b});
    return b;
}
}  // namespace

void destroy_batch_state(S2Context* ctx) {
    std::lock_guard<std::mutex> lock(g_registry_mutex);
    for (size_t i = 0; i < g_registry.items.size(); ++i) {
        if (g_registry.items[i].first != ctx) continue;
        BatchState* b = g_registry.items[i].second;
        free_bufs(b->qbufs);
        free_bufs(b->pbufs);
        if (b->done_host) cudaFreeHost(b->done_host);
        delete b;
        g_registry.items.erase(g_registry.items.begin() + i);
        return;
    }
}
}  // namespace s2

extern "C" int s2_render_views(S2Context* ctx, const S2View* views, uint32_t nviews, const S2RenderParams* prm,
                               const S2Aovs* outs, int out_on_host, S2RenderStats* stats_out) {
    using namespace s2;
    if (!ctx) return S2_ERR_INVALID;
    if (!views || !prm || nviews == 0) return set_error(ctx, S2_ERR_INVALID, "views, view count and params are required");
    if (nviews > 255) return set_error(ctx, S2_ERR_INVALID, "at most 255 views per call");
    if (!ctx->has_bvh) return set_error(ctx, S2_ERR_NO_SCENE, "s2_render_views before s2_scene_upload + s2_build_bvh");
    if (prm->spp == 0) return set_error(ctx, S2_ERR_INVALID, "spp must be >= 1");
    if (prm->max_path_length > 255) return set_error(ctx, S2_ERR_INVALID, "max_path_length must be <= 255");
    if ((prm->flags & S2_FLAG_RESTIR_DI) && (prm->restir_candidates == 0 || prm->restir_candidates > 1024))
        return set_error(ctx, S2_ERR_INVALID, "restir_candidates must be in 1..1024");
    if ((prm->flags & S2_FLAG_RESTIR_REUSE) && (prm->flags & S2_FLAG_RESTIR_SCREEN))
        return set_error(ctx, S2_ERR_INVALID, "S2_FLAG_RESTIR_REUSE and S2_FLAG_RESTIR_SCREEN are exclusive");
    const bool screen = (prm->flags & S2_FLAG_RESTIR_DI) && (prm->flags & S2_FLAG_RESTIR_SCREEN);
    if (screen && (prm->flags & S2_FLAG_RADIANCE_CACHE))
        return set_error(ctx, S2_ERR_UNSUPPORTED, "batched screen-space ReSTIR reuse takes no radiance cache");
    if (screen && (prm->restir_spatial > 32 || !(prm->restir_spatial_radius >= 0.f) || !std::isfinite(prm->restir_spatial_radius) ||
                   !(prm->restir_max_m > 0.f)))
        return set_error(ctx, S2_ERR_INVALID, "invalid screen-space ReSTIR parameters (restir_spatial <= 32, "
                                              "restir_spatial_radius >= 0, restir_max_m > 0)");
    const bool reuse = (prm->flags & S2_FLAG_RESTIR_DI) && (prm->flags & S2_FLAG_RESTIR_REUSE);
    if (reuse && (prm->restir_grid_cells > (1u << 26) || prm->restir_grid_cell_size < 0.f ||
                  !std::isfinite(prm->restir_grid_cell_size) || !(prm->restir_grid_pixel_radius >= 0.f) ||
                  !std::isfinite(prm->restir_grid_pixel_radius) || !(prm->restir_max_m > 0.f)))
        return set_error(ctx, S2_ERR_INVALID, "invalid ReSTIR hash-grid parameters");
    const bool cache = (prm->flags & S2_FLAG_RADIANCE_CACHE) != 0;
    if (cache && !ctx->cache) return set_error(ctx, S2_ERR_INVALID, "S2_FLAG_RADIANCE_CACHE needs s2_cache_init");
    // radiance cache: training paths are extra paths after the views' (their own accumulators)
    const uint32_t train_paths = cache ? (prm->cache_train_paths ? prm->cache_train_paths : 65536u) : 0u;
    cudaSetDevice(ctx->device);
    std::vector<ViewEntry> ve(nviews);
    std::vector<uint32_t> layout;
    uint64_t pixels = 0, paths = 0;
    for (uint32_t v = 0; v < nviews; ++v) {
        const S2View& V = views[v];
        const int W = V.image_max[0] - V.image_min[0], H = V.image_max[1] - V.image_min[1];
        if (W <= 0 || H <= 0 || (int64_t)W * H > (1ll << 28)) return set_error(ctx, S2_ERR_INVALID, "invalid extent of view " + std::to_string(v));
        ViewEntry& e = ve[v];
        std::memset(&e, 0, sizeof(e));
        std::memcpy(e.proj, V.projection, sizeof(e.proj));
        e.imin[0] = V.image_min[0]; e.imin[1] = V.image_min[1]; e.imax[0] = V.image_max[0]; e.imax[1] = V.image_max[1];
        std::memcpy(e.cam, V.camera_to_world, sizeof(e.cam));
        std::memcpy(e.prev_inv, V.prev_world_to_camera, sizeof(e.prev_inv));
        e.width = (uint32_t)W; e.height = (uint32_t)H; e.pixels = (uint32_t)(W * H);
        e.pixel_offset = (uint32_t)pixels;
        e.path_offset = paths;
        pixels += e.pixels;
        paths += (uint64_t)e.pixels * prm->spp;
        layout.push_back((uint32_t)W); layout.push_back((uint32_t)H);
    }
    if (pixels > (1ull << 30)) return set_error(ctx, S2_ERR_INVALID, "too many pixels in one call");
    BatchState* B = g_batch_for(ctx);
    if (!B) return set_error(ctx, S2_ERR_OOM, "batch state allocation failed");
    cudaStream_t s = ctx->stream;
    const uint64_t wave = prm->wave_paths ? prm->wave_paths : (ctx->tuning.wave_paths ? ctx->tuning.wave_paths : kDefaultWavePaths);
    const uint32_t capacity = (uint32_t)std::max<uint64_t>(1024, std::min<uint64_t>(wave, paths + train_paths));
    if (B->capacity < capacity) {
        free_bufs(B->qbufs);
        B->capacity = 0;
        for (int k = 0; k < 2; ++k) {
            B->q[k].s0 = (float4*)dev_alloc(ctx, B->qbufs, 16ull * capacity);
            B->q[k].s1 = (float4*)dev_alloc(ctx, B->qbufs, 16ull * capacity);
            B->q[k].s2 = (float4*)dev_alloc(ctx, B->qbufs, 16ull * capacity);
            B->q[k].s3 = (uint4*)dev_alloc(ctx, B->qbufs, 16ull * capacity);
        }
        B->hits = (float4*)dev_alloc(ctx, B->qbufs, 16ull * capacity);
        B->sh_o = (float4*)dev_alloc(ctx, B->qbufs, 16ull * capacity);
        B->sh_d = (float4*)dev_alloc(ctx, B->qbufs, 16ull * capacity);
        B->sh_c = (float4*)dev_alloc(ctx, B->qbufs, 16ull * capacity);
        if (B->qbufs.size() != 12) { free_bufs(B->qbufs); return S2_ERR_OOM; }
        B->capacity = capacity;
    }
    const bool relayout = B->layout != layout || B->views_cap < nviews;
    if (relayout) {
        free_bufs(B->pbufs);
        B->total_fx = (unsigned long long*)dev_alloc(ctx, B->pbufs, 32ull * pixels);
        B->views_dev = (ViewEntry*)dev_alloc(ctx, B->pbufs, sizeof(ViewEntry) * 256);
        B->stream_state = (unsigned long long*)dev_alloc(ctx, B->pbufs, 64);
        B->counters = (uint32_t*)dev_alloc(ctx, B->pbufs, sizeof(uint32_t) * C_COUNT);
        B->stats = (unsigned long long*)dev_alloc(ctx, B->pbufs, sizeof(unsigned long long) * S_COUNT);
        B->stage_rad = (float4*)dev_alloc(ctx, B->pbufs, 16ull * pixels);
        if (B->pbufs.size() != 6) { free_bufs(B->pbufs); B->layout.clear(); return S2_ERR_OOM; }
        if (!B->done_host && cudaMallocHost(&B->done_host, 64) != cudaSuccess) { cudaGetLastError(); return set_error(ctx, S2_ERR_OOM, "pinned allocation failed"); }
        B->layout = layout;
        B->views_cap = 256;
        B->pixels = pixels;
        B->accumulated_spp = 0;
        cudaMemsetAsync(B->total_fx, 0, 32ull * pixels, s);
    }
    // AOV outputs: device pointers directly, or staged per view for host outputs
    std::vector<DevBuf> stage;
    for (uint32_t v = 0; v < nviews; ++v) {
        if (!outs) break;
        const S2Aovs& o = outs[v];
        ViewEntry& e = ve[v];
        auto pick = [&](void* user, size_t elem) -> void* {
            if (!user) return nullptr;
            if (!out_on_host) return user;
            return dev_alloc(ctx, stage, elem * e.pixels);
        };
        e.aov_albedo = (float4*)pick(o.albedo, 16);
        e.aov_vis = (uint2*)pick(o.visibility, 8);
        e.aov_depth = (float4*)pick(o.depth, 16);
        e.aov_prev_uv = (float2*)pick(o.prev_uv, 8);
        e.aov_ids = (uint2*)pick(o.ids32, 8);
    }
    cudaMemcpyAsync(B->views_dev, ve.data(), sizeof(ViewEntry) * nviews, cudaMemcpyHostToDevice, s);
    if (!(prm->flags & S2_FLAG_ACCUMULATE)) {
        cudaMemsetAsync(B->total_fx, 0, 32ull * pixels, s);
        B->accumulated_spp = 0;
    }
    cudaMemsetAsync(B->stream_state, 0, 64, s);
    cudaMemsetAsync(B->counters, 0, sizeof(uint32_t) * C_COUNT, s);
    cudaMemsetAsync(B->stats, 0, sizeof(unsigned long long) * S_COUNT, s);
    cudaMemsetAsync(ctx->status_dev, 0, sizeof(int), s);

    PTParams P;
    std::memset(&P, 0, sizeof(P));
    P.scene = ctx->scene;
    if (ctx->tuning.shade_records == S2_SHADE_RECORDS_OFF) P.scene.shade_recs = nullptr;
    P.scene.light_power_pick = (prm->flags & S2_FLAG_LIGHT_POWER_PICK) ? 1u : 0u;
    P.scene.env_fp_on = (prm->flags & S2_FLAG_ENV_FOOTPRINT_PDF) ? 1u : 0u;
    P.scene.env_sample_prob = prm->environment_sample_probability > 0.f ? prm->environment_sample_probability : 0.9f;
    P.min_len = prm->min_path_length;
    P.max_len = prm->max_path_length;
    P.flags = prm->flags;
    P.frame_seed = prm->frame_seed;
    P.restir_m = prm->restir_candidates ? prm->restir_candidates : 32;
    P.trav.tris_per_step = ctx->tuning.trav_tris_per_step;
    P.trav.vote8 = ctx->tuning.trav_vote8;
    P.refill_min = ctx->tuning.refill_min;
    const bool sort = ctx->tuning.shade_order == S2_SHADE_ORDER_MATERIAL;
    P.exposure = prm->exposure;
    P.q[0] = B->q[0]; P.q[1] = B->q[1];
    P.hits = B->hits; P.sh_o = B->sh_o; P.sh_d = B->sh_d; P.sh_c = B->sh_c;
    P.counters = B->counters;
    P.stats = B->stats;
    P.status = ctx->status_dev;
    P.views = B->views_dev;
    P.nviews = nviews;
    P.view_spp = prm->spp;
    P.total_fx = B->total_fx;
    P.total_paths = paths + train_paths;
    P.image_paths = paths;
    P.batch_pixels = (uint32_t)pixels;
    P.capacity = capacity;
    P.stream_state = B->stream_state;
    P.pixels = 1;  // unused in batched mode

    RenderState* st = ctx->render;
    if (!st) {
        int rc = ensure_state(ctx, 1, 1, 1);  // occupancy-derived grid sizes
        if (rc != S2_OK) return rc;
        st = ctx->render;
    }
    if (sort) {
        const int rc = ensure_sort(ctx, st, capacity);
        if (rc != S2_OK) return set_error(ctx, rc, "material-sort buffer allocation failed");
        P.sort_on = 1; P.sort_keys = st->sort_keys; P.sort_perm = st->sort_perm; P.sort_hist = st->sort_hist;
    }
    if (reuse) {
        // ReSTIR DI hash-grid reuse across the views of the call, as TestRenderer renders all its
        // views into one world-space grid (TestRenderer.cpp:488-493): the grid holds
        // pixels x min(2, maxDepth-1) records per sample pass over all views, and its cell sizes
        // follow view 0's camera.  This call appends to one grid of the pair and reads the other,
        // the previous call's (s2_render's grids: either entry point continues the sequence).
        const uint32_t cells = prm->restir_grid_cells ? prm->restir_grid_cells : 100000u;
        const uint64_t per_pass = (uint64_t)pixels * std::max(1u, std::min(2u, prm->max_path_length ? prm->max_path_length - 1 : 1u));
        const uint32_t size = (uint32_t)std::min<uint64_t>(per_pass * prm->spp, 1u << 24);
        RenderState::Grid& cur = st->grid[st->grid_cur];
        RenderState::Grid& prev = st->grid[st->grid_cur ^ 1];
        const int rc = ensure_grid(ctx, cur, cells, size);
        if (rc != S2_OK) return set_error(ctx, rc, "hash grid allocation failed");
        HashGridDev& g = cur.g;
        const S2View& v0 = views[0];
        const int W0 = v0.image_max[0] - v0.image_min[0], H0 = v0.image_max[1] - v0.image_min[1];
        g.min_cell_size = prm->restir_grid_cell_size > 0.f ? prm->restir_grid_cell_size : 0.5f;
        g.cell_pixel_radius = prm->restir_grid_pixel_radius;
        g.camera_position = make_float3(v0.camera_to_world[3], v0.camera_to_world[7], v0.camera_to_world[11]);
        g.distance_scale = tanf(g.cell_pixel_radius * v0.projection[7] *
                                std::max(1.f / (float)H0, (float)H0 / ((float)W0 * (float)W0)));
        cudaMemsetAsync(g.checksums, 0, sizeof(uint32_t) * cells, s);
        cudaMemsetAsync(g.cell_counters, 0, sizeof(uint32_t) * cells, s);
        cudaMemsetAsync(g.other, 0, sizeof(uint32_t) * 4, s);
        P.grid_cur = g;
        P.grid_prev = prev.g;
        P.prev_valid = st->grid_prev_valid && prev.g.checksums ? 1u : 0u;
        P.reuse = 1;
        P.max_m = prm->restir_max_m;
    } else {
        st->grid_prev_valid = false;  // a call without reuse drops the grids, as s2_render does
    }
    if (screen) {
        // one reservoir per pixel of every view (views at their pixel offsets), kept for the next
        // call with the same view layout
        uint32_t key = 2166136261u;  // FNV-1a of the view extents
        for (uint32_t x : layout) { key ^= x; key *= 16777619u; }
        key |= 0x80000000u;
        if (st->ss_pixels != (uint32_t)pixels || st->ss_width != key) {
            free_bufs(st->ss_bufs);
            st->ss_pixels = 0;
            st->ss_prev_valid = false;
            st->ss[0] = (ReservoirRecord*)dev_alloc(ctx, st->ss_bufs, sizeof(ReservoirRecord) * pixels);
            st->ss[1] = (ReservoirRecord*)dev_alloc(ctx, st->ss_bufs, sizeof(ReservoirRecord) * pixels);
            if (!st->ss[0] || !st->ss[1]) { free_bufs(st->ss_bufs); return set_error(ctx, S2_ERR_OOM, "reservoir buffer allocation failed"); }
            st->ss_pixels = (uint32_t)pixels;
            st->ss_width = key;
        }
        ReservoirRecord* cur = st->ss[st->ss_cur];
        cudaMemsetAsync(cur, 0, sizeof(ReservoirRecord) * pixels, s);
        P.ss_on = 1;
        P.ss_cur = cur;
        P.ss_prev = st->ss[st->ss_cur ^ 1u];
        P.ss_prev_valid = st->ss_prev_valid ? 1u : 0u;
        P.ss_spatial = prm->restir_spatial ? prm->restir_spatial : 5u;
        P.ss_radius = prm->restir_spatial_radius > 0.f ? prm->restir_spatial_radius : 30.f;
        P.max_m = prm->restir_max_m;
    } else {
        st->ss_prev_valid = false;
    }
    if (cache) {
        // terminal-vertex queries of one iteration (at most a queue) and the training vertices of the
        // call; training paths accumulate into train_accum (zeroed per call)
        const uint64_t tr_cap64 = std::min<uint64_t>((uint64_t)train_paths * std::max(1u, prm->max_path_length), 1u << 26);
        int rc = ensure_cache_queues(ctx, st, capacity, (uint32_t)tr_cap64);
        if (rc != S2_OK) return set_error(ctx, rc, "radiance cache queue allocation failed");
        if (B->train_cap < train_paths) {
            free_bufs(B->tbufs);
            B->train_cap = 0;
            B->train_accum = (float4*)dev_alloc(ctx, B->tbufs, sizeof(float4) * (size_t)train_paths);
            if (!B->train_accum) return set_error(ctx, S2_ERR_OOM, "training accumulator allocation failed");
            B->train_cap = train_paths;
        }
        cudaMemsetAsync(B->train_accum, 0, sizeof(float4) * (size_t)train_paths, s);
        cache_prepare_device(ctx);  // kernel attributes, outside the graph capture
        P.accum = B->train_accum;
        P.cache_on = 1;
        P.cache_len = (prm->cache_bounces ? prm->cache_bounces : 2u) + 1u;
        P.cache_rough = std::min(1.f, std::max(0.f, prm->cache_min_roughness));
        P.cq_pos = st->cq_pos; P.cq_thr = st->cq_thr; P.cq_cap = st->cq_cap;
        P.tr_pos = st->tr_pos; P.tr_thr = st->tr_thr; P.tr_rad = st->tr_rad; P.tr_cap = st->tr_cap;
    }
    const bool lam = (prm->flags & S2_FLAG_LAMBERTIAN) != 0, restir = (prm->flags & S2_FLAG_RESTIR_DI) != 0;
    const bool count = (prm->flags & S2_FLAG_COUNT_FETCHES) != 0;
    int apply_rc = S2_OK;
    // one graph = two iterations (parity 0 and 1) of setup, regeneration, extend, [material sort,]
    // shade, [radiance-cache inference for the terminal vertices,] occlude; with shadow merging
    // (not with the cache) each iteration's k_trace also traces the previous iteration's shadow
    // rays, whose count sits in the other parity's counter.  The iteration whose setup finds no
    // path left still traces the last shadow rays before the host sees it done.
    const bool merge = !cache && ctx->tuning.shadow_merge != S2_SHADOW_MERGE_OFF;
    P.sh_merge = merge ? 1u : 0u;
    auto iteration = [&](uint32_t parity, int first) {
        P.sh_parity = merge ? parity : 0u;
        const uint32_t sh_prev = parity ? C_SHADOW : C_SHADOW1;  // counter of parity 1 - parity
        k_stream_setup<<<1, 32, 0, s>>>(P, parity, first);
        k_regen<<<std::min<uint32_t>((capacity + 255) / 256, 148u * 16u), 256, 0, s>>>(P, parity);
        if (merge && !first) {
            if (count) k_trace<true><<<st->ext_blocks, kTravBlock, 0, s>>>(P, parity, sh_prev);
            else k_trace<false><<<st->ext_blocks, kTravBlock, 0, s>>>(P, parity, sh_prev);
        } else {
            if (count) k_extend<true><<<st->ext_blocks, kTravBlock, 0, s>>>(P, parity);
            else k_extend<false><<<st->ext_blocks, kTravBlock, 0, s>>>(P, parity);
        }
        if (sort) launch_sort(P, parity, st->sort_blocks, s);
        if (lam) { if (restir) launch_shade<true, true>(P, parity, st, s); else launch_shade<true, false>(P, parity, st, s); }
        else { if (restir) launch_shade<false, true>(P, parity, st, s); else launch_shade<false, false>(P, parity, st, s); }
        if (cache) {
            const int r = cache_apply_device(ctx, st->cq_pos, st->cq_thr, st->cq_cap, B->counters + C_CACHEQ, nullptr, B->total_fx);
            if (r != S2_OK) apply_rc = r;
        }
        if (!merge) {
            if (count) k_occlude<true><<<st->occ_blocks, kTravBlock, 0, s>>>(P);
            else k_occlude<false><<<st->occ_blocks, kTravBlock, 0, s>>>(P);
        }
    };
    cudaEventRecord(ctx->ev0, s);
    iteration(0, 1);  // first iteration outside the graph (it skips the shadow accounting)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int rc = check_cuda(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    if (rc != S2_OK) return rc;
    iteration(1, 0);
    iteration(0, 0);
    rc = check_cuda(ctx, cudaStreamEndCapture(s, &graph), "cudaStreamEndCapture");
    if (rc == S2_OK) rc = check_cuda(ctx, cudaGraphInstantiate(&exec, graph, 0), "cudaGraphInstantiate");
    if (rc != S2_OK) { if (graph) cudaGraphDestroy(graph); return rc; }
    if (apply_rc != S2_OK) { cudaGraphExecDestroy(exec); cudaGraphDestroy(graph); return apply_rc; }
    const uint64_t per_iter = (sort ? 8 : 5) + (cache ? 1 : 0) - (merge ? 1 : 0);
    uint64_t launches = per_iter;
    // replay until the device reports every path finished; the check trails one group behind so
    // the host never waits on the group it just queued
    const uint64_t lower = (paths + train_paths + capacity - 1) / capacity;
    const uint64_t cap_iters = (paths + train_paths) * (uint64_t)std::max(1u, prm->max_path_length) / std::max<uint64_t>(1, capacity) +
                               prm->max_path_length + 4;
    const uint32_t group = 4;  // graph launches (8 iterations) per done check
    uint64_t iters = 1;
    cudaEvent_t pending = nullptr;
    cudaEventCreateWithFlags(&pending, cudaEventDisableTiming);
    bool done = false, have_pending = false;
    while (!done && iters < cap_iters + 2) {
        for (uint32_t g = 0; g < group; ++g) { cudaGraphLaunch(exec, s); iters += 2; launches += 2 * per_iter; }
        if (have_pending) {
            cudaEventSynchronize(pending);
            done = *B->done_host != 0;
        }
        if (iters >= lower) {
            cudaMemcpyAsync(B->done_host, B->stream_state + 3, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
            cudaEventRecord(pending, s);
            have_pending = true;
        }
    }
    cudaStreamSynchronize(s);
    cudaEventDestroy(pending);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (!*B->done_host) return set_error(ctx, S2_ERR_DEVICE, "batched render did not finish within its iteration bound");
    if (reuse) {
        // GpuHashGrid::build (GpuHashGrid.cpp:84-111), then this grid becomes the previous one
        launches += build_grid(ctx, st->grid[st->grid_cur], s);
        st->grid_cur ^= 1u;
        st->grid_prev_valid = true;
    }
    if (cache) {
        // online training on this call's training paths (as after each wave of s2_render)
        k_cache_targets<<<std::max(1, st->shade_blocks / 2), 256, 0, s>>>(P);
        rc = cache_backward_device(ctx, st->tr_pos, st->tr_rad, st->tr_cap, B->counters + C_TRAIN);
        if (rc == S2_OK) rc = cache_adam_device(ctx, st->tr_cap, B->counters + C_TRAIN);
        if (rc != S2_OK) return rc;
        launches += 4;
    }
    if (screen) {  // this call's reservoirs become the previous ones
        st->ss_cur ^= 1u;
        st->ss_prev_valid = true;
    }
    B->accumulated_spp += prm->spp;
    const float scale = (float)(1.0 / (double)B->accumulated_spp) * exp2f(prm->exposure);
    for (uint32_t v = 0; v < nviews; ++v) {
        float4* dst = (outs && outs[v].radiance && !out_on_host) ? (float4*)outs[v].radiance : B->stage_rad + ve[v].pixel_offset;
        k_resolve_fx<<<(ve[v].pixels + 255) / 256, 256, 0, s>>>(B->total_fx, ve[v].pixel_offset, ve[v].pixels, scale, dst);
        launches++;
    }
    cudaEventRecord(ctx->ev1, s);
    rc = check_cuda(ctx, cudaGetLastError(), "batched render");
    if (rc != S2_OK) { free_bufs(stage); return rc; }
    if (out_on_host && outs) {
        for (uint32_t v = 0; v < nviews; ++v) {
            const S2Aovs& o = outs[v];
            const ViewEntry& e = ve[v];
            if (o.radiance) cudaMemcpyAsync(o.radiance, B->stage_rad + e.pixel_offset, 16ull * e.pixels, cudaMemcpyDeviceToHost, s);
            if (o.albedo) cudaMemcpyAsync(o.albedo, e.aov_albedo, 16ull * e.pixels, cudaMemcpyDeviceToHost, s);
            if (o.visibility) cudaMemcpyAsync(o.visibility, e.aov_vis, 8ull * e.pixels, cudaMemcpyDeviceToHost, s);
            if (o.depth) cudaMemcpyAsync(o.depth, e.aov_depth, 16ull * e.pixels, cudaMemcpyDeviceToHost, s);
            if (o.prev_uv) cudaMemcpyAsync(o.prev_uv, e.aov_prev_uv, 8ull * e.pixels, cudaMemcpyDeviceToHost, s);
            if (o.ids32) cudaMemcpyAsync(o.ids32, e.aov_ids, 8ull * e.pixels, cudaMemcpyDeviceToHost, s);
        }
    }
    unsigned long long sv[S_COUNT] = {0, 0, 0, 0, 0, 0, 0, 0};
    int status = 0;
    cudaMemcpyAsync(sv, B->stats, sizeof(sv), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&status, ctx->status_dev, sizeof(int), cudaMemcpyDeviceToHost, s);
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "batched render");
    free_bufs(stage);
    if (rc != S2_OK) return rc;
    if (status & 4) return set_error(ctx, S2_ERR_TIMEOUT, "tensor-core wait timed out in the radiance cache");
    if (status) return set_error(ctx, S2_ERR_DEVICE, "traversal stack overflow during render");
    if (stats_out) {
        std::memset(stats_out, 0, sizeof(*stats_out));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        stats_out->extension_rays = sv[S_EXT];
        stats_out->shadow_rays = sv[S_SHADOW];
        stats_out->paths = paths;
        stats_out->nan_count = sv[S_NAN];
        stats_out->gpu_ms = ms;
        stats_out->kernel_launches = launches;
        stats_out->extend_node_fetches = sv[S_EXT_NODES];
        stats_out->extend_tri_fetches = sv[S_EXT_TRIS];
        stats_out->shadow_node_fetches = sv[S_SH_NODES];
        stats_out->shadow_tri_fetches = sv[S_SH_TRIS];
    }
    return S2_OK;
}

// ============================================================================== tuning
extern "C" int s2_set_tuning(S2Context* ctx, const S2Tuning* t) {
    if (!ctx) return S2_ERR_INVALID;
    if (!t) { std::memset(&ctx->tuning, 0, sizeof(ctx->tuning)); return S2_OK; }
    if (t->trav_tris_per_step > 32 || t->trav_vote8 > 9 || t->refill_min > 32 || (t->wave_paths && t->wave_paths < 1024) ||
        t->shade_order > S2_SHADE_ORDER_QUEUE || t->trace_order > S2_TRACE_ORDER_COHERENT ||
        t->shade_records > S2_SHADE_RECORDS_OFF || t->shadow_merge > S2_SHADOW_MERGE_OFF)
        return set_error(ctx, S2_ERR_INVALID, "tuning out of range (tris_per_step <= 32, vote8 <= 9, refill_min <= 32, "
                                              "wave_paths 0 or >= 1024, shade_order, trace_order, shade_records and "
                                              "shadow_merge 0 or 1)");
    ctx->tuning = *t;
    return S2_OK;
}

extern "C" int s2_get_tuning(S2Context* ctx, S2Tuning* t) {
    if (!ctx || !t) return S2_ERR_INVALID;
    *t = ctx->tuning;
    return S2_OK;
}

extern "C" int s2_autotune(S2Context* ctx, const S2View* view, const S2RenderParams* prm, S2Tuning* out,
                           uint32_t* trials_out) {
    if (!ctx) return S2_ERR_INVALID;
    if (!view || !prm) return set_error(ctx, S2_ERR_INVALID, "view and params are required");
    S2RenderParams p = *prm;
    p.flags &= ~(S2_FLAG_ACCUMULATE | S2_FLAG_PROFILE_KERNELS | S2_FLAG_COUNT_FETCHES);
    p.wave_paths = 0;
    const S2Tuning saved = ctx->tuning;
    uint32_t trials = 0;
    uint32_t seed = p.frame_seed;
    // ray throughput of the current tuning: best of two renders (the first also warms caches)
    auto measure = [&](double& mrays) -> int {
        double best = 0.0;
        for (int k = 0; k < 2; ++k) {
            p.frame_seed = seed;
            seed += std::max(1u, p.spp);
            S2RenderStats st;
            const int rc = s2_render(ctx, view, &p, nullptr, 0, &st);
            if (rc != S2_OK) return rc;
            trials++;
            if (st.gpu_ms > 0) best = std::max(best, (double)(st.extension_rays + st.shadow_rays) / st.gpu_ms / 1e3);
        }
        mrays = best;
        return S2_OK;
    };
    S2Tuning best = saved;
    double best_rate = 0.0;
    int rc = measure(best_rate);
    if (rc != S2_OK) { ctx->tuning = saved; return rc; }
    const uint32_t waves[] = {1u << 23, 1u << 24, 1u << 25, 1u << 26, 1u << 27};
    const uint32_t tris[] = {1, 2, 4, 8};
    const uint32_t votes[] = {2, 3, 4, 5, 6};
    const uint32_t refills[] = {4, 8, 12, 16};
    const uint32_t sorts[] = {S2_SHADE_ORDER_MATERIAL, S2_SHADE_ORDER_QUEUE};
    const uint32_t traces[] = {S2_TRACE_ORDER_QUEUE, S2_TRACE_ORDER_COHERENT};
    const uint32_t merges[] = {S2_SHADOW_MERGE_ON, S2_SHADOW_MERGE_OFF};
    for (int pass = 0; pass < 2; ++pass) {
        for (int knob = 0; knob < 7; ++knob) {
            const uint32_t* vals = knob == 0 ? waves : knob == 1 ? tris : knob == 2 ? votes : knob == 3 ? refills
                                 : knob == 4 ? sorts : knob == 5 ? traces : merges;
            const int nv = knob == 0 ? 5 : knob == 1 ? 4 : knob == 2 ? 5 : knob == 3 ? 4 : 2;
            for (int v = 0; v < nv; ++v) {
                S2Tuning t = best;
                uint32_t* field = knob == 0 ? &t.wave_paths : knob == 1 ? &t.trav_tris_per_step
                                : knob == 2 ? &t.trav_vote8 : knob == 3 ? &t.refill_min : knob == 4 ? &t.shade_order
                                : knob == 5 ? &t.trace_order : &t.shadow_merge;
                if (*field == vals[v]) continue;
                *field = vals[v];
                ctx->tuning = t;
                double rate = 0.0;
                rc = measure(rate);
                if (rc != S2_OK) { ctx->tuning = saved; return rc; }
                if (rate > best_rate * 1.01) { best_rate = rate; best = t; }
            }
        }
    }
    ctx->tuning = best;
    if (out) *out = best;
    if (trials_out) *trials_out = trials;
    return S2_OK;
}
