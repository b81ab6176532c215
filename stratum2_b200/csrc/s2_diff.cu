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
        return set_error(ctx, S2_ERR_INVALID, "pixels x spp must stay below 2^32 (one thread per path)");
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

template <bool ADJ>
void launch(const DiffArgs& A, cudaStream_t s) {
    const uint32_t blocks = (uint32_t)(((uint64_t)A.pixels * A.spp + 127) / 128);
    if (A.flags & S2_FLAG_LAMBERTIAN) dk::k_diff<true, ADJ><<<blocks, 128, 0, s>>>(A);
    else dk::k_diff<false, ADJ><<<blocks, 128, 0, s>>>(A);
    if (!ADJ) dk::k_diff_resolve<<<(A.pixels + 255) / 256, 256, 0, s>>>(A);
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
    cudaMemsetAsync(A.rays, 0, 2 * sizeof(unsigned long long), ctx->stream);
    cudaMemsetAsync(ctx->status_dev, 0, sizeof(int), ctx->stream);
    cudaEventRecord(ctx->ev0, ctx->stream);
    launch<false>(A, ctx->stream);
    rc = check_cuda(ctx, cudaGetLastError(), "differentiable render launch");
    if (rc != S2_OK) { cudaStreamSynchronize(ctx->stream); free_bufs(tmp); return rc; }
    if (out_on_host) cudaMemcpyAsync(radiance, A.image, sizeof(float4) * A.pixels, cudaMemcpyDeviceToHost, ctx->stream);
    return finish(ctx, tmp, A.rays, 0.f, stats_out, (uint64_t)A.pixels * A.spp, 2);
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
    if (!A.rays || !A.grad || !A.grad_offset || !A.d_image) { free_bufs(tmp); return S2_ERR_OOM; }
    cudaMemcpyAsync((void*)A.grad_offset, off.data(), sizeof(uint32_t) * (ni + 1), cudaMemcpyHostToDevice, ctx->stream);
    if (on_host) cudaMemcpyAsync((void*)A.d_image, d_radiance, sizeof(float4) * A.pixels, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemsetAsync(A.grad, 0, sizeof(float4) * std::max<size_t>(1, off[ni]), ctx->stream);
    cudaMemsetAsync(A.rays, 0, 2 * sizeof(unsigned long long), ctx->stream);
    cudaMemsetAsync(ctx->status_dev, 0, sizeof(int), ctx->stream);
    cudaEventRecord(ctx->ev0, ctx->stream);
    launch<true>(A, ctx->stream);
    rc = check_cuda(ctx, cudaGetLastError(), "adjoint render launch");
    if (rc != S2_OK) { cudaStreamSynchronize(ctx->stream); free_bufs(tmp); return rc; }
    for (uint32_t k = 0; k < ni; ++k) {
        if (!d_images[k]) continue;
        const size_t bytes = sizeof(float4) * (size_t)(off[k + 1] - off[k]);
        cudaMemcpyAsync(d_images[k], A.grad + off[k], bytes, on_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                        ctx->stream);
    }
    return finish(ctx, tmp, A.rays, 0.f, stats_out, (uint64_t)A.pixels * A.spp, 1);
}
