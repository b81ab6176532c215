// Differentiable rendering entry points (s2_render_diff, s2_render_adjoint); no counterpart in the
// reference.  Kernels in s2_diff.cuh.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "s2_context.h"

// The renderer's device code, compiled here with internal linkage (inside an unnamed namespace,
// its namespace renamed) so the header-defined kernels do not collide with s2_render.cu's.
#define s2 s2_diff_impl
namespace {
#include "s2_diff.cuh"
}  // namespace
#undef s2
namespace dk = s2_diff_impl;
using dk::DiffArgs;
using s2::DevBuf;
using s2::check_cuda;
using s2::dev_alloc;
using s2::free_bufs;
using s2::set_error;

namespace {

constexpr uint32_t kDiffUnsupported = S2_FLAG_RESTIR_DI | S2_FLAG_RESTIR_REUSE | S2_FLAG_RESTIR_SCREEN | S2_FLAG_RADIANCE_CACHE | S2_FLAG_ACCUMULATE |
                                      S2_FLAG_PROFILE_KERNELS | S2_FLAG_COUNT_FETCHES;

int check_args(S2Context* ctx, const S2View* view, const S2RenderParams* prm, DiffArgs& A) {
    if (!view || !prm) return set_error(ctx, S2_ERR_INVALID, "view and params are required");
    if (!ctx->has_bvh) return set_error(ctx, S2_ERR_NO_SCENE, "differentiable render before s2_scene_upload + s2_build_bvh");
    const int W = view->image_max[0] - view->image_min[0], H = view->image_max[1] - view->image_min[1];
    if (W <= 0 || H <= 0 || (int64_t)W * H > (1ll << 26)) return set_error(ctx, S2_ERR_INVALID, "invalid view extent");
    if (prm->spp == 0) return set_error(ctx, S2_ERR_INVALID, "spp must be >= 1");
    if ((uint64_t)W * H * prm->spp > 0xffffffffull)
        return set_error(ctx, S2_ERR_INVALID, "pixels x spp must stay below 2^32 (32-bit path ids)");
    if (prm->max_path_length > 255) return set_error(ctx, S2_ERR_INVALID, "max_path_length must be <= 255");
    if (prm->flags & kDiffUnsupported)
        return set_error(ctx, S2_ERR_UNSUPPORTED, "differentiable rendering supports plain NEE path tracing only "
                                                  "(no ReSTIR, radiance cache, accumulation or profiling flags)");
    std::memset(&A, 0, sizeof(A));
    A.scene = ctx->scene;
    A.scene.light_power_pick = (prm->flags & S2_FLAG_LIGHT_POWER_PICK) ? 1u : 0u;
    A.scene.env_fp_on = (prm->flags & S2_FLAG_ENV_FOOTPRINT_PDF) ? 1u : 0u;
    A.scene.env_sample_prob = prm->environment_sample_probability > 0.f ? prm->environment_sample_probability : 0.9f;
    std::memcpy(A.proj, view->projection, sizeof(A.proj));
    A.imin[0] = view->image_min[0]; A.imin[1] = view->image_min[1];
    A.imax[0] = view->image_max[0]; A.imax[1] = view->image_max[1];
    std::memcpy(A.cam, view->camera_to_world, sizeof(A.cam));
    A.width = (uint32_t)W; A.height = (uint32_t)H; A.pixels = (uint32_t)W * (uint32_t)H;
    A.spp = prm->spp;
    A.min_len = prm->min_path_length;
    A.max_len = prm->max_path_length;
    A.flags = prm->flags;
    A.frame_seed = prm->frame_seed;
    A.out_scale = exp2f(prm->exposure) / (float)prm->spp;
    A.status = ctx->status_dev;
    return S2_OK;
}

// Wavefront buffers of one call: paths are rendered in waves of at most kDiffWave.
constexpr uint32_t kDiffWave = 1u << 23;

struct DiffWave {
    dk::PTParams P;
    dk::DiffQueues Q;
    uint32_t cap = 0;
    int ext_blocks = 0, shade_blocks = 0, occ_blocks = 0, grad_blocks = 0;
};

// adjoint: also the visibility words of every path and the gradient records of one bounce
int alloc_wave(S2Context* ctx, std::vector<DevBuf>& tmp, const DiffArgs& A, DiffWave& w, bool adjoint) {
    const uint64_t total = (uint64_t)A.pixels * A.spp;
    w.cap = (uint32_t)std::min<uint64_t>(total, kDiffWave);
    std::memset(&w.P, 0, sizeof(w.P));
    std::memset(&w.Q, 0, sizeof(w.Q));
    w.Q.paths = (uint32_t)total;
    w.P.sh_o = (float4*)dev_alloc(ctx, tmp, sizeof(float4) * (size_t)w.cap);
    w.P.sh_d = (float4*)dev_alloc(ctx, tmp, sizeof(float4) * (size_t)w.cap);
    w.P.sh_c = (float4*)dev_alloc(ctx, tmp, sizeof(float4) * (size_t)w.cap);
    w.Q.gcount = (uint32_t*)dev_alloc(ctx, tmp, sizeof(uint32_t));
    if (!w.P.sh_o || !w.P.sh_d || !w.P.sh_c || !w.Q.gcount) return S2_ERR_OOM;
    if (adjoint) {
        // at most three records per vertex: an environment hit, or NEE (material + environment)
        // and the continuation
        w.Q.vis = (uint32_t*)dev_alloc(ctx, tmp, sizeof(uint32_t) * total * ((A.max_len + 31u) >> 5));
        w.Q.grec = (float4*)dev_alloc(ctx, tmp, sizeof(float4) * 9 * (size_t)w.cap);
        if (!w.Q.vis || !w.Q.grec) return S2_ERR_OOM;
    }
    w.P.scene = A.scene;
    if (ctx->tuning.shade_records == S2_SHADE_RECORDS_OFF) w.P.scene.shade_recs = nullptr;
    w.P.flags = A.flags;
    w.P.trav.tris_per_step = ctx->tuning.trav_tris_per_step;
    w.P.trav.vote8 = ctx->tuning.trav_vote8;
    w.P.refill_min = ctx->tuning.refill_min;
    w.P.status = A.status;
    for (int k = 0; k < 2; ++k) {
        // positional: the four 16-byte streams of a path queue (the namespace rename above also
        // renames the queue's third member)
        float4* a = (float4*)dev_alloc(ctx, tmp, sizeof(float4) * (size_t)w.cap);
        float4* b = (float4*)dev_alloc(ctx, tmp, sizeof(float4) * (size_t)w.cap);
        float4* c = (float4*)dev_alloc(ctx, tmp, sizeof(float4) * (size_t)w.cap);
        uint4* d = (uint4*)dev_alloc(ctx, tmp, sizeof(uint4) * (size_t)w.cap);
        if (adjoint) w.Q.L[k] = (float4*)dev_alloc(ctx, tmp, sizeof(float4) * (size_t)w.cap);
        if (!a || !b || !c || !d || (adjoint && !w.Q.L[k])) return S2_ERR_OOM;
        w.P.q[k] = dk::PathQueue{a, b, c, d};
    }
    w.P.hits = (float4*)dev_alloc(ctx, tmp, sizeof(float4) * (size_t)w.cap);
    w.P.counters = (uint32_t*)dev_alloc(ctx, tmp, sizeof(uint32_t) * dk::C_COUNT);
    w.P.stats = (unsigned long long*)dev_alloc(ctx, tmp, sizeof(unsigned long long) * dk::S_COUNT);
    if (!w.P.hits || !w.P.counters || !w.P.stats) return S2_ERR_OOM;
    int sms = 148, b = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, dk::k_extend<false>, dk::kTravBlock, 0);
    w.ext_blocks = std::max(1, b) * sms;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (A.flags & S2_FLAG_LAMBERTIAN) ? dk::k_diff_shade<true> : dk::k_diff_shade<false>,
                                                  128, 0);
    w.shade_blocks = std::max(1, b) * sms;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, dk::k_diff_occlude, dk::kTravBlock, 0);
    w.occ_blocks = std::max(1, b) * sms;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (A.flags & S2_FLAG_LAMBERTIAN) ? dk::k_diff_grads<true> : dk::k_diff_grads<false>,
                                                  128, 0);
    w.grad_blocks = std::max(1, b) * sms;
    return S2_OK;
}

// Renders every path in waves (adj: the second replay, path_l holding each path's radiance).
// Returns the kernel launches issued.
uint64_t launch(const DiffArgs& A, DiffWave& w, bool adj, cudaStream_t s) {
    const uint64_t total = (uint64_t)A.pixels * A.spp;
    const uint32_t bounces = std::max(1u, A.max_len);
    uint64_t launches = 0;
    for (uint64_t base = 0; base < total; base += w.cap) {
        const uint32_t n = (uint32_t)std::min<uint64_t>(w.cap, total - base);
        cudaMemsetAsync(w.P.counters, 0, sizeof(uint32_t) * dk::C_COUNT, s);
        dk::k_diff_gen<<<(n + 255) / 256, 256, 0, s>>>(A, w.P, w.Q, (uint32_t)base, n, adj ? 1 : 0);
        launches += 1;
        const bool lambert = (A.flags & S2_FLAG_LAMBERTIAN) != 0;
        for (uint32_t b = 0; b < bounces; ++b) {
            const uint32_t parity = b & 1u;
            dk::k_diff_bounce<<<1, 32, 0, s>>>(A, w.P, w.Q, parity);
            dk::k_extend<false><<<w.ext_blocks, dk::kTravBlock, 0, s>>>(w.P, parity);
            if (lambert) dk::k_diff_shade<true><<<w.shade_blocks, 128, 0, s>>>(A, w.P, w.Q, parity, adj ? 1 : 0);
            else dk::k_diff_shade<false><<<w.shade_blocks, 128, 0, s>>>(A, w.P, w.Q, parity, adj ? 1 : 0);
            // the forward traces the bounce's shadow rays; the adjoint replay pushes its gradients
            if (!adj) dk::k_diff_occlude<<<w.occ_blocks, dk::kTravBlock, 0, s>>>(A, w.P, w.Q);
            else if (lambert) dk::k_diff_grads<true><<<w.grad_blocks, 128, 0, s>>>(A, w.Q);
            else dk::k_diff_grads<false><<<w.grad_blocks, 128, 0, s>>>(A, w.Q);
            launches += 4;
        }
    }
    if (!adj) {
        dk::k_diff_resolve<<<(A.pixels + 255) / 256, 256, 0, s>>>(A);
        launches += 1;
    }
    return launches;
}

int finish(S2Context* ctx, std::vector<DevBuf>& tmp, unsigned long long* rays_dev, float ms_unused, S2RenderStats* st,
           uint64_t paths, uint64_t launches) {
    (void)ms_unused;
    unsigned long long rays[2] = {0, 0};
    int status = 0;
    cudaMemcpyAsync(rays, rays_dev, sizeof(rays), cudaMemcpyDeviceToHost, ctx->stream);
    cudaMemcpyAsync(&status, ctx->status_dev, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    cudaEventRecord(ctx->ev1, ctx->stream);
    int rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "differentiable render");
    float ms = 0.f;
    if (rc == S2_OK) cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    free_bufs(tmp);
    if (rc != S2_OK) return rc;
    if (status) return set_error(ctx, S2_ERR_DEVICE, "traversal stack overflow during differentiable render");
    if (st) {
        std::memset(st, 0, sizeof(*st));
        st->extension_rays = rays[0];
        st->shadow_rays = rays[1];
        st->paths = paths;
        st->gpu_ms = ms;
        st->kernel_launches = launches;
    }
    return S2_OK;
}

}  // namespace

extern "C" int s2_render_diff(S2Context* ctx, const S2View* view, const S2RenderParams* prm, float* radiance, int out_on_host,
                              S2RenderStats* stats_out) {
    if (!ctx) return S2_ERR_INVALID;
    DiffArgs A;
    int rc = check_args(ctx, view, prm, A);
    if (rc != S2_OK) return rc;
    if (!radiance) return set_error(ctx, S2_ERR_INVALID, "radiance output is required");
    cudaSetDevice(ctx->device);
    std::vector<DevBuf> tmp;
    A.rays = (unsigned long long*)dev_alloc(ctx, tmp, 2 * sizeof(unsigned long long));
    A.image = out_on_host ? (float4*)dev_alloc(ctx, tmp, sizeof(float4) * A.pixels) : (float4*)radiance;
    A.path_l = (float4*)dev_alloc(ctx, tmp, sizeof(float4) * (size_t)A.pixels * A.spp);
    if (!A.rays || !A.image || !A.path_l) { free_bufs(tmp); return S2_ERR_OOM; }
    DiffWave w;
    if (alloc_wave(ctx, tmp, A, w, false) != S2_OK) { free_bufs(tmp); return set_error(ctx, S2_ERR_OOM, "differentiable render queues"); }
    cudaMemsetAsync(A.rays, 0, 2 * sizeof(unsigned long long), ctx->stream);
    cudaMemsetAsync(ctx->status_dev, 0, sizeof(int), ctx->stream);
    cudaEventRecord(ctx->ev0, ctx->stream);
    const uint64_t launches = launch(A, w, false, ctx->stream);
    rc = check_cuda(ctx, cudaGetLastError(), "differentiable render launch");
    if (rc != S2_OK) { cudaStreamSynchronize(ctx->stream); free_bufs(tmp); return rc; }
    if (out_on_host) cudaMemcpyAsync(radiance, A.image, sizeof(float4) * A.pixels, cudaMemcpyDeviceToHost, ctx->stream);
    return finish(ctx, tmp, A.rays, 0.f, stats_out, (uint64_t)A.pixels * A.spp, launches);
}

extern "C" int s2_render_adjoint(S2Context* ctx, const S2View* view, const S2RenderParams* prm, const float* d_radiance,
                                 int on_host, float* const* d_images, S2RenderStats* stats_out) {
    if (!ctx) return S2_ERR_INVALID;
    DiffArgs A;
    int rc = check_args(ctx, view, prm, A);
    if (rc != S2_OK) return rc;
    if (!d_radiance || !d_images) return set_error(ctx, S2_ERR_INVALID, "d_radiance and d_images are required");
    cudaSetDevice(ctx->device);
    const uint32_t ni = (uint32_t)ctx->images_host.size();
    std::vector<uint32_t> off(ni + 1, 0);
    for (uint32_t k = 0; k < ni; ++k) {
        const uint64_t next = (uint64_t)off[k] + (uint64_t)ctx->images_host[k].width * ctx->images_host[k].height;
        if (next > 0xffffffffull) return set_error(ctx, S2_ERR_INVALID, "images too large for gradients");
        off[k + 1] = (uint32_t)next;
    }
    std::vector<DevBuf> tmp;
    A.rays = (unsigned long long*)dev_alloc(ctx, tmp, 2 * sizeof(unsigned long long));
    A.grad = (float4*)dev_alloc(ctx, tmp, sizeof(float4) * std::max<size_t>(1, off[ni]));
    A.grad_offset = (const uint32_t*)dev_alloc(ctx, tmp, sizeof(uint32_t) * (ni + 1));
    A.d_image = on_host ? (const float4*)dev_alloc(ctx, tmp, sizeof(float4) * A.pixels) : (const float4*)d_radiance;
    A.path_l = (float4*)dev_alloc(ctx, tmp, sizeof(float4) * (size_t)A.pixels * A.spp);
    A.image = (float4*)dev_alloc(ctx, tmp, sizeof(float4) * A.pixels);
    if (!A.rays || !A.grad || !A.grad_offset || !A.d_image || !A.path_l || !A.image) { free_bufs(tmp); return S2_ERR_OOM; }
    DiffWave w;
    if (alloc_wave(ctx, tmp, A, w, true) != S2_OK) { free_bufs(tmp); return set_error(ctx, S2_ERR_OOM, "adjoint render queues"); }
    cudaMemcpyAsync((void*)A.grad_offset, off.data(), sizeof(uint32_t) * (ni + 1), cudaMemcpyHostToDevice, ctx->stream);
    if (on_host) cudaMemcpyAsync((void*)A.d_image, d_radiance, sizeof(float4) * A.pixels, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemsetAsync(A.grad, 0, sizeof(float4) * std::max<size_t>(1, off[ni]), ctx->stream);
    cudaMemsetAsync(A.rays, 0, 2 * sizeof(unsigned long long), ctx->stream);
    cudaMemsetAsync(ctx->status_dev, 0, sizeof(int), ctx->stream);
    cudaEventRecord(ctx->ev0, ctx->stream);
    // first replay: every path's radiance into path_l; second replay: the texel gradients
    uint64_t launches = launch(A, w, false, ctx->stream);
    launches += launch(A, w, true, ctx->stream);
    rc = check_cuda(ctx, cudaGetLastError(), "adjoint render launch");
    if (rc != S2_OK) { cudaStreamSynchronize(ctx->stream); free_bufs(tmp); return rc; }
    for (uint32_t k = 0; k < ni; ++k) {
        if (!d_images[k]) continue;
        const size_t bytes = sizeof(float4) * (size_t)(off[k + 1] - off[k]);
        cudaMemcpyAsync(d_images[k], A.grad + off[k], bytes, on_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                        ctx->stream);
    }
    return finish(ctx, tmp, A.rays, 0.f, stats_out, (uint64_t)A.pixels * A.spp, launches);
}
