// Learned radiance cache: parameters, optimiser state and the C ABI (s2_cache_*).  No counterpart
// in the reference; the kernels are in s2_cache.cuh.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "s2_cache.cuh"
#include "s2_context.h"

namespace s2 {

struct CacheState {
    S2CacheParams prm{};
    uint32_t table_entries = 0;      // levels * 2^log2_table
    std::vector<DevBuf> bufs;
    float* w32 = nullptr;            // f32 master weights (S2_CACHE_WEIGHTS)
    float* t32 = nullptr;            // f32 master table (entries * 2)
    __half2* t16 = nullptr;          // f16 table used by the kernels
    uint4* wimage = nullptr;         // f16 weights in the tensor-core operand layout
    float* adam_w = nullptr;         // m, v for the weights (2 * S2_CACHE_WEIGHTS)
    float* adam_t = nullptr;         // m, v for the table (2 * entries * 2)
    float* grad_w = nullptr;         // weight gradient accumulator
    float* grad_t = nullptr;         // table gradient accumulator
    uint64_t step = 0;
    CacheDev dev{};
    int sms = 148;
};

void destroy_cache_state(S2Context* ctx) {
    if (!ctx->cache) return;
    free_bufs(ctx->cache->bufs);
    delete ctx->cache;
    ctx->cache = nullptr;
}

namespace {

// f16 copies of the parameters: the table as half2 and the weights as the byte image of the three
// K-major operand tiles (W1 64 x 32, W2 64 x 64, W3 padded to 16 x 64).
__global__ void k_cache_pack(const float* __restrict__ w32, const float* __restrict__ t32, __half2* __restrict__ t16,
                             uint32_t entries, uint8_t* __restrict__ wimage) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < entries) t16[i] = __floats2half2_rn(t32[2 * i], t32[2 * i + 1]);
    if (i < kCacheW1) {
        const uint32_t o = i / kCacheIn, k = i % kCacheIn;
        *(__half*)(wimage + kmaj_offset(o, k, kCacheIn)) = __float2half_rn(w32[i]);
    }
    if (i < kCacheW2) {
        const uint32_t o = i / kCacheHidden, k = i % kCacheHidden;
        *(__half*)(wimage + kW1Bytes + kmaj_offset(o, k, kCacheHidden)) = __float2half_rn(w32[kCacheW1 + i]);
    }
    if (i < kCacheOutPad * kCacheHidden) {
        const uint32_t o = i / kCacheHidden, k = i % kCacheHidden;
        const float v = o < kCacheOut ? w32[kCacheW1 + kCacheW2 + i] : 0.f;
        *(__half*)(wimage + kW1Bytes + kW2Bytes + kmaj_offset(o, k, kCacheHidden)) = __float2half_rn(v);
    }
}

uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
float uniform(uint64_t& s, float lo, float hi) {
    return lo + (hi - lo) * (float)((splitmix(s) >> 40) * (1.0 / 16777216.0));
}

int repack(S2Context* ctx) {
    CacheState* c = ctx->cache;
    const uint32_t n = std::max(c->table_entries, kCacheW2);
    k_cache_pack<<<(n + 255) / 256, 256, 0, ctx->stream>>>(c->w32, c->t32, c->t16, c->table_entries, (uint8_t*)c->wimage);
    return check_cuda(ctx, cudaGetLastError(), "cache pack");
}

}  // namespace
}  // namespace s2

using namespace s2;

extern "C" void s2_cache_default_params(S2CacheParams* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->log2_table = 19;
    p->base_resolution = 16;
    p->max_resolution = 2048;
    p->learning_rate = 1e-2f;
    p->beta1 = 0.9f;
    p->beta2 = 0.99f;
    p->epsilon = 1e-15f;
    p->seed = 1337;
}

extern "C" int s2_cache_init(S2Context* ctx, const S2CacheParams* params) {
    if (!ctx) return S2_ERR_INVALID;
    S2CacheParams p;
    s2_cache_default_params(&p);
    if (params) p = *params;
    if (p.log2_table < 8 || p.log2_table > 24) return set_error(ctx, S2_ERR_INVALID, "log2_table must be in 8..24");
    if (p.base_resolution < 1 || p.max_resolution < p.base_resolution || p.max_resolution > (1u << 20))
        return set_error(ctx, S2_ERR_INVALID, "invalid cache resolutions");
    bool box_ok = true;
    for (int k = 0; k < 3; ++k) box_ok = box_ok && std::isfinite(p.box_min[k]) && std::isfinite(p.box_max[k]) && p.box_max[k] > p.box_min[k];
    if (!box_ok) {
        if (!ctx->has_scene) return set_error(ctx, S2_ERR_NO_SCENE, "cache box not given and no scene uploaded");
        const float4 sp = ctx->scene.scene_sphere;
        const float c3[3] = {sp.x, sp.y, sp.z};
        for (int k = 0; k < 3; ++k) { p.box_min[k] = c3[k] - sp.w; p.box_max[k] = c3[k] + sp.w; }
    }
    cudaSetDevice(ctx->device);
    destroy_cache_state(ctx);
    CacheState* c = ctx->cache = new (std::nothrow) CacheState();
    if (!c) return set_error(ctx, S2_ERR_OOM, "cache state allocation failed");
    c->prm = p;
    c->table_entries = kCacheLevels << p.log2_table;
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const size_t ne = c->table_entries;
    c->w32 = (float*)dev_alloc(ctx, c->bufs, sizeof(float) * kCacheWeights);
    c->t32 = (float*)dev_alloc(ctx, c->bufs, sizeof(float) * 2 * ne);
    c->t16 = (__half2*)dev_alloc(ctx, c->bufs, sizeof(__half2) * ne);
    c->wimage = (uint4*)dev_alloc(ctx, c->bufs, kWImageBytes);
    c->adam_w = (float*)dev_alloc(ctx, c->bufs, sizeof(float) * 2 * kCacheWeights);
    c->adam_t = (float*)dev_alloc(ctx, c->bufs, sizeof(float) * 4 * ne);
    c->grad_w = (float*)dev_alloc(ctx, c->bufs, sizeof(float) * kCacheWeights);
    c->grad_t = (float*)dev_alloc(ctx, c->bufs, sizeof(float) * 2 * ne);
    for (auto& b : c->bufs) if (!b.ptr) { destroy_cache_state(ctx); return set_error(ctx, S2_ERR_OOM, "cache allocation failed"); }
    if (c->bufs.size() != 8) { destroy_cache_state(ctx); return set_error(ctx, S2_ERR_OOM, "cache allocation failed"); }
    // initial parameters
    uint64_t rs = 0x5eedull ^ ((uint64_t)p.seed << 17);
    std::vector<float> w(kCacheWeights), t(2 * ne);
    const uint32_t fan[3][2] = {{kCacheIn, kCacheHidden}, {kCacheHidden, kCacheHidden}, {kCacheHidden, kCacheOut}};
    const uint32_t off[4] = {0, kCacheW1, kCacheW1 + kCacheW2, kCacheWeights};
    for (int l = 0; l < 3; ++l) {
        const float a = std::sqrt(6.f / (float)(fan[l][0] + fan[l][1]));
        for (uint32_t i = off[l]; i < off[l + 1]; ++i) w[i] = uniform(rs, -a, a);
    }
    for (size_t i = 0; i < t.size(); ++i) t[i] = uniform(rs, -1e-4f, 1e-4f);
    return s2_cache_set_params(ctx, w.data(), t.data());
}

extern "C" int s2_cache_set_params(S2Context* ctx, const float* weights, const float* table) {
    if (!ctx) return S2_ERR_INVALID;
    CacheState* c = ctx->cache;
    if (!c) return set_error(ctx, S2_ERR_NO_SCENE, "s2_cache_set_params before s2_cache_init");
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const size_t ne = c->table_entries;
    if (weights) cudaMemcpyAsync(c->w32, weights, sizeof(float) * kCacheWeights, cudaMemcpyHostToDevice, s);
    if (table) cudaMemcpyAsync(c->t32, table, sizeof(float) * 2 * ne, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(c->adam_w, 0, sizeof(float) * 2 * kCacheWeights, s);
    cudaMemsetAsync(c->adam_t, 0, sizeof(float) * 4 * ne, s);
    cudaMemsetAsync(c->grad_w, 0, sizeof(float) * kCacheWeights, s);
    cudaMemsetAsync(c->grad_t, 0, sizeof(float) * 2 * ne, s);
    c->step = 0;
    int rc = repack(ctx);
    if (rc != S2_OK) return rc;
    // device view used by the kernels
    CacheDev& d = c->dev;
    d.table = c->t16;
    d.log2_table = c->prm.log2_table;
    const double b = kCacheLevels > 1 ? std::exp((std::log((double)c->prm.max_resolution) - std::log((double)c->prm.base_resolution)) /
                                                 (double)(kCacheLevels - 1)) : 1.0;
    for (uint32_t l = 0; l < kCacheLevels; ++l) {
        d.res[l] = (float)std::floor((double)c->prm.base_resolution * std::pow(b, (double)l) + 1e-9);
        const double cells = std::pow((double)d.res[l] + 1.0, 3.0);
        d.dense[l] = cells <= (double)(1u << c->prm.log2_table) ? 1u : 0u;
    }
    d.box_min = make_float3(c->prm.box_min[0], c->prm.box_min[1], c->prm.box_min[2]);
    d.box_inv_extent = make_float3(1.f / (c->prm.box_max[0] - c->prm.box_min[0]), 1.f / (c->prm.box_max[1] - c->prm.box_min[1]),
                                   1.f / (c->prm.box_max[2] - c->prm.box_min[2]));
    d.wimage = c->wimage;
    d.status = ctx->status_dev;
    return check_cuda(ctx, cudaStreamSynchronize(s), "cache parameter upload");
}

extern "C" int s2_cache_get_params(S2Context* ctx, float* weights, float* table) {
    if (!ctx) return S2_ERR_INVALID;
    CacheState* c = ctx->cache;
    if (!c) return set_error(ctx, S2_ERR_NO_SCENE, "s2_cache_get_params before s2_cache_init");
    cudaSetDevice(ctx->device);
    if (weights) cudaMemcpyAsync(weights, c->w32, sizeof(float) * kCacheWeights, cudaMemcpyDeviceToHost, ctx->stream);
    if (table) cudaMemcpyAsync(table, c->t32, sizeof(float) * 2 * (size_t)c->table_entries, cudaMemcpyDeviceToHost, ctx->stream);
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "cache parameter download");
}

namespace s2 {
// Launches the inference kernel for n float4 positions already on the device.
int cache_infer_device(S2Context* ctx, const float4* pos, uint32_t n, float4* out) {
    CacheState* c = ctx->cache;
    if (n == 0) return S2_OK;
    static bool attr_set[64] = {};
    if (ctx->device < 64 && !attr_set[ctx->device]) {
        cudaFuncSetAttribute(k_cache_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInfSmemBytes);
        attr_set[ctx->device] = true;
    }
    const uint32_t tiles = (n + kCacheTile - 1) / kCacheTile;
    const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)c->sms);
    k_cache_infer<<<grid, 128, kInfSmemBytes, ctx->stream>>>(c->dev, pos, n, out);
    return check_cuda(ctx, cudaGetLastError(), "cache inference launch");
}
}  // namespace s2

extern "C" int s2_cache_query(S2Context* ctx, const float* positions, uint32_t n, float* radiance, int on_device) {
    if (!ctx) return S2_ERR_INVALID;
    if (!ctx->cache) return set_error(ctx, S2_ERR_NO_SCENE, "s2_cache_query before s2_cache_init");
    if (n == 0) return S2_OK;
    if (!positions || !radiance) return set_error(ctx, S2_ERR_INVALID, "positions/radiance is null");
    cudaSetDevice(ctx->device);
    std::vector<DevBuf> tmp;
    const float4* dpos = (const float4*)positions;
    float4* dout = (float4*)radiance;
    if (!on_device) {
        dpos = (const float4*)dev_alloc(ctx, tmp, sizeof(float4) * (size_t)n);
        dout = (float4*)dev_alloc(ctx, tmp, sizeof(float4) * (size_t)n);
        if (!dpos || !dout) { free_bufs(tmp); return S2_ERR_OOM; }
        cudaMemcpyAsync((void*)dpos, positions, sizeof(float4) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream);
    }
    cudaMemsetAsync(ctx->status_dev, 0, sizeof(int), ctx->stream);
    int rc = cache_infer_device(ctx, dpos, n, dout);
    int status = 0;
    if (rc == S2_OK) {
        if (!on_device) cudaMemcpyAsync(radiance, dout, sizeof(float4) * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream);
        cudaMemcpyAsync(&status, ctx->status_dev, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
        rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "cache query");
    }
    cudaStreamSynchronize(ctx->stream);
    free_bufs(tmp);
    if (rc == S2_OK && (status & 4)) rc = set_error(ctx, S2_ERR_TIMEOUT, "tensor-core wait timed out in cache inference");
    return rc;
}
