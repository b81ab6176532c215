// s2_render_noalloc: the wavefront path tracer without any device allocation.
//
// Some callers cannot allocate device memory when they render: a host application that owns the
// GPU's memory budget and forbids allocation once its frame loop runs (cudaMalloc / cudaFree also
// synchronise the whole device, which a real-time frame cannot absorb), or an embedding plugin
// that may only use the buffers its host hands it.  For them this entry point renders with the
// same kernels as s2_render, but takes its scratch -- the path queues, hit records, shadow-ray
// queue, per-path accumulators and counters -- from one file-scope device array of fixed size,
// and accumulates radiance directly in the caller's output buffer.  It calls no cudaMalloc,
// cudaFree or allocating library routine.
//
// Limits and behaviour:
//  * The array is S2_NOALLOC_SCRATCH_BYTES (64 MiB) and lives on every GPU that loads the library
//    until the process exits.  A wave holds whole images, so an image may have at most
//    S2_NOALLOC_MAX_PIXELS pixels; larger views are rejected with S2_ERR_INVALID.
//  * The first call on a device looks up the array's device address (cudaGetSymbolAddress, with
//    that device current) and caches it; make that first call before any stream capture.
//  * All calls share the array, which keeps the previous call's contents; each call clears what
//    must start at zero.  Calls whose GPU work overlaps (other streams, other host threads) race
//    on the array: serialise them.
//  * Outputs are device pointers; the radiance buffer is required.  S2_FLAG_ACCUMULATE and
//    S2_FLAG_PROFILE_KERNELS are rejected (they need state or events this variant does not keep),
//    and so are the modes that need buffers of their own: ReSTIR reuse, the radiance cache and
//    light tracing.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "s2_context.h"

// The kernels of s2_render, compiled here with internal linkage (inside an unnamed namespace,
// their namespace renamed) so this file shares their code without touching s2_render's.
#define s2 s2_noalloc_impl
namespace {
#include "s2_shade_kernel.cuh"
}  // namespace
#undef s2
namespace nak = s2_noalloc_impl;

#define S2_NOALLOC_SCRATCH_BYTES (64ull << 20)
#define S2_NOALLOC_HEADER_BYTES 4096ull
// per path: two path queues (2 x 64 B), hit (16 B), shadow ray (48 B), accumulator (16 B), in 13
// streams of 16 bytes per path, each stream's start rounded up to 256 bytes
#define S2_NOALLOC_PATH_BYTES 208ull
#define S2_NOALLOC_STREAMS 13ull
#define S2_NOALLOC_MAX_PIXELS \
    ((S2_NOALLOC_SCRATCH_BYTES - S2_NOALLOC_HEADER_BYTES - 256ull * S2_NOALLOC_STREAMS) / S2_NOALLOC_PATH_BYTES)
static_assert(S2_NOALLOC_MAX_PIXELS == 322603ull, "documented pixel limit of s2_render_noalloc");

static __device__ __align__(256) unsigned char g_noalloc_scratch[S2_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};
int g_blocks[kMaxDevices][4] = {};  // persistent grid sizes: extend, occlude, shade, ReSTIR shade

// Once per device, with that device current: the device address of the scratch array and the
// occupancy-derived grid sizes.
int noalloc_setup(S2Context* ctx, unsigned char** scratch, int blocks[4]) {
    if (ctx->device < 0 || ctx->device >= kMaxDevices) return s2::set_error(ctx, S2_ERR_UNSUPPORTED, "device index too large");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[ctx->device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return s2::set_error(ctx, S2_ERR_CUDA, std::string("cudaGetSymbolAddress of the scratch array failed: ") +
                                                       cudaGetErrorString(e));
        }
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess)
            return s2::set_error(ctx, S2_ERR_CUDA, "cudaGetDeviceProperties failed");
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, nak::k_extend<false>, nak::kTravBlock, 0);
        g_blocks[ctx->device][0] = std::max(1, b) * prop.multiProcessorCount;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, nak::k_occlude<false>, nak::kTravBlock, 0);
        g_blocks[ctx->device][1] = std::max(1, b) * prop.multiProcessorCount;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, nak::k_shade<false, false>, 128, 0);
        g_blocks[ctx->device][2] = std::max(1, b) * prop.multiProcessorCount;
        // the ReSTIR variants keep more state live and are compiled for fewer blocks per SM
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, nak::k_shade<false, true>, 128, 0);
        g_blocks[ctx->device][3] = std::max(1, b) * prop.multiProcessorCount;
        g_scratch_ptr[ctx->device] = (unsigned char*)p;
    }
    *scratch = g_scratch_ptr[ctx->device];
    std::memcpy(blocks, g_blocks[ctx->device], sizeof(int) * 4);
    return S2_OK;
}

// in-place mean and exposure of the accumulated radiance
__global__ void k_noalloc_scale(float4* __restrict__ rad, uint32_t pixels, float scale) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pixels) return;
    const float4 t = rad[p];
    rad[p] = make_float4(t.x * scale, t.y * scale, t.z * scale, 1.f);
}

}  // namespace

extern "C" int s2_render_noalloc(S2Context* ctx, const S2View* view, const S2RenderParams* prm, const S2Aovs* out,
                                 S2RenderStats* stats_out) {
    using namespace nak;
    using s2::check_cuda;
    using s2::set_error;
    if (!ctx) return S2_ERR_INVALID;
    if (!view || !prm || !out || !out->radiance)
        return set_error(ctx, S2_ERR_INVALID, "s2_render_noalloc: view, params and a device radiance buffer are required");
    if (!ctx->has_bvh) return set_error(ctx, S2_ERR_NO_SCENE, "s2_render_noalloc before s2_scene_upload + s2_build_bvh");
    if (prm->flags & (S2_FLAG_ACCUMULATE | S2_FLAG_PROFILE_KERNELS))
        return set_error(ctx, S2_ERR_INVALID, "s2_render_noalloc does not support S2_FLAG_ACCUMULATE or S2_FLAG_PROFILE_KERNELS");
    const int W = view->image_max[0] - view->image_min[0], H = view->image_max[1] - view->image_min[1];
    if (W <= 0 || H <= 0) return set_error(ctx, S2_ERR_INVALID, "invalid view extent");
    const uint64_t pixels64 = (uint64_t)W * (uint64_t)H;
    if (pixels64 > S2_NOALLOC_MAX_PIXELS)
        return set_error(ctx, S2_ERR_INVALID, "s2_render_noalloc: " + std::to_string(pixels64) +
                                                  " pixels exceed the scratch limit of " +
                                                  std::to_string(S2_NOALLOC_MAX_PIXELS) + " pixels (64 MiB scratch array)");
    if (prm->spp == 0) return set_error(ctx, S2_ERR_INVALID, "spp must be >= 1");
    if (prm->max_path_length > 255) return set_error(ctx, S2_ERR_INVALID, "max_path_length must be <= 255");
    if (prm->flags & (S2_FLAG_RESTIR_REUSE | S2_FLAG_RESTIR_SCREEN | S2_FLAG_RADIANCE_CACHE | S2_FLAG_LIGHT_TRACE))
        return set_error(ctx, S2_ERR_UNSUPPORTED, "S2_FLAG_RESTIR_REUSE, S2_FLAG_RESTIR_SCREEN, S2_FLAG_RADIANCE_CACHE and "
                                                  "S2_FLAG_LIGHT_TRACE are supported by s2_render only");
    if ((prm->flags & S2_FLAG_RESTIR_DI) && (prm->restir_candidates == 0 || prm->restir_candidates > 1024))
        return set_error(ctx, S2_ERR_INVALID, "restir_candidates must be in 1..1024");
    cudaSetDevice(ctx->device);
    unsigned char* scratch = nullptr;
    int blocks[4];
    int rc = noalloc_setup(ctx, &scratch, blocks);
    if (rc != S2_OK) return rc;
    cudaStream_t s = ctx->stream;

    const uint32_t pixels = (uint32_t)pixels64;
    const uint64_t target = prm->wave_paths ? prm->wave_paths : (ctx->tuning.wave_paths ? ctx->tuning.wave_paths : (1u << 22));
    const uint64_t max_paths = std::min<uint64_t>(target, S2_NOALLOC_MAX_PIXELS);
    const uint32_t slots = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(prm->spp, max_paths / pixels));
    const size_t cap = (size_t)slots * pixels;

    // carve the scratch array: counters and stats first, then per-path streams
    uint32_t* counters = (uint32_t*)scratch;
    unsigned long long* stats = (unsigned long long*)(scratch + 256);
    unsigned char* cur = scratch + S2_NOALLOC_HEADER_BYTES;
    auto take = [&](size_t bytes) { unsigned char* p = cur; cur += (bytes + 255) & ~size_t(255); return p; };

    PTParams P;
    std::memset(&P, 0, sizeof(P));
    for (int k = 0; k < 2; ++k) {
        // positional: the four 16-byte streams of a path queue
        float4* a = (float4*)take(16 * cap);
        float4* b = (float4*)take(16 * cap);
        float4* c = (float4*)take(16 * cap);
        uint4* d = (uint4*)take(16 * cap);
        P.q[k] = nak::PathQueue{a, b, c, d};
    }
    P.hits = (float4*)take(16 * cap);
    P.sh_o = (float4*)take(16 * cap);
    P.sh_d = (float4*)take(16 * cap);
    P.sh_c = (float4*)take(16 * cap);
    P.accum = (float4*)take(16 * cap);
    if ((uint64_t)(cur - scratch) > S2_NOALLOC_SCRATCH_BYTES)
        return set_error(ctx, S2_ERR_INVALID, "s2_render_noalloc: wave does not fit the scratch array");

    P.scene = ctx->scene;
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
    P.trav.tris_per_step = ctx->tuning.trav_tris_per_step;  // traversal tuning, as s2_render takes it
    P.trav.vote8 = ctx->tuning.trav_vote8;
    P.refill_min = ctx->tuning.refill_min;
    P.counters = counters;
    P.stats = stats;
    P.status = ctx->status_dev;
    P.aov_albedo = (float4*)out->albedo;
    P.aov_vis = (uint2*)out->visibility;
    P.aov_depth = (float4*)out->depth;
    P.aov_prev_uv = (float2*)out->prev_uv;
    P.aov_ids = (uint2*)out->ids32;
    float4* rad = (float4*)out->radiance;

    // the shared array keeps the previous call's contents: clear what must start at zero
    cudaMemsetAsync(scratch, 0, S2_NOALLOC_HEADER_BYTES, s);
    cudaMemsetAsync(P.accum, 0, 16 * cap, s);
    cudaMemsetAsync(rad, 0, sizeof(float4) * pixels, s);
    cudaMemsetAsync(ctx->status_dev, 0, sizeof(int), s);
    cudaEventRecord(ctx->ev0, s);
    const bool lam = (prm->flags & S2_FLAG_LAMBERTIAN) != 0, restir = (prm->flags & S2_FLAG_RESTIR_DI) != 0;
    const bool count = (prm->flags & S2_FLAG_COUNT_FETCHES) != 0;
    uint64_t launches = 0;
    for (uint32_t done = 0; done < prm->spp; done += slots) {
        P.wave_base_sample = done;
        P.wave_samples = std::min(slots, prm->spp - done);
        const uint32_t n = P.wave_samples * pixels;
        k_raygen<<<(n + 255) / 256, 256, 0, s>>>(P);
        for (uint32_t b = 0; b < prm->max_path_length; ++b) {
            const uint32_t parity = b & 1u;
            k_bounce_setup<<<1, 32, 0, s>>>(P, parity, b == 0);
            if (count) k_extend<true><<<blocks[0], kTravBlock, 0, s>>>(P, parity);
            else k_extend<false><<<blocks[0], kTravBlock, 0, s>>>(P, parity);
            if (lam) {
                if (restir) k_shade<true, true><<<blocks[3], 128, 0, s>>>(P, parity);
                else k_shade<true, false><<<blocks[2], 128, 0, s>>>(P, parity);
            } else {
                if (restir) k_shade<false, true><<<blocks[3], 128, 0, s>>>(P, parity);
                else k_shade<false, false><<<blocks[2], 128, 0, s>>>(P, parity);
            }
            if (count) k_occlude<true><<<blocks[1], kTravBlock, 0, s>>>(P);
            else k_occlude<false><<<blocks[1], kTravBlock, 0, s>>>(P);
            launches += 4;
        }
        k_wave_finish<<<1, 32, 0, s>>>(P);
        k_reduce<<<(pixels + 255) / 256, 256, 0, s>>>(P, rad);  // accumulate into the caller's buffer
        launches += 3;
    }
    k_noalloc_scale<<<(pixels + 255) / 256, 256, 0, s>>>(rad, pixels, (float)(1.0 / (double)prm->spp) * exp2f(prm->exposure));
    launches += 1;
    cudaEventRecord(ctx->ev1, s);
    rc = check_cuda(ctx, cudaGetLastError(), "s2_render_noalloc kernel launch");
    if (rc != S2_OK) return rc;
    unsigned long long sv[S_COUNT] = {0, 0, 0, 0, 0, 0, 0, 0};
    int status = 0;
    cudaMemcpyAsync(sv, stats, sizeof(sv), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&status, ctx->status_dev, sizeof(int), cudaMemcpyDeviceToHost, s);
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "s2_render_noalloc");
    if (rc != S2_OK) return rc;
    if (status) return set_error(ctx, S2_ERR_DEVICE, "traversal stack overflow during render");
    if (stats_out) {
        std::memset(stats_out, 0, sizeof(*stats_out));
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
    }
    return S2_OK;
}
