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
    float* loss = nullptr;           // summed per-record loss of the last pass
    uint64_t step = 0;
    uint32_t inject_wait_polls = 0;  // armed by s2_inject_wait_timeout for the next inference launch
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
    if (i < entries) t16[i] = __floats2half2_rn(t32[2 * i], t32[2 * i + 1]);  // entries = 0: weights only
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
    // transposed copies: W2T (i, o) = W2[o][i], W1T (i, o) = W1[o][i]
    if (i < kCacheW2) {
        const uint32_t o = i / kCacheHidden, k = i % kCacheHidden;
        *(__half*)(wimage + kWImageBytes + kmaj_offset(k, o, kCacheHidden)) = __float2half_rn(w32[kCacheW1 + i]);
    }
    if (i < kCacheW1) {
        const uint32_t o = i / kCacheIn, k = i % kCacheIn;
        *(__half*)(wimage + kWImageBytes + kW2TBytes + kmaj_offset(k, o, kCacheHidden)) = __float2half_rn(w32[i]);
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

int repack(S2Context* ctx, bool table = true) {
    CacheState* c = ctx->cache;
    const uint32_t entries = table ? c->table_entries : 0u;
    const uint32_t n = std::max(entries, kCacheW2);
    k_cache_pack<<<(n + 255) / 256, 256, 0, ctx->stream>>>(c->w32, c->t32, c->t16, entries, (uint8_t*)c->wimage);
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
    c->wimage = (uint4*)dev_alloc(ctx, c->bufs, kWImageTrainBytes);
    c->loss = (float*)dev_alloc(ctx, c->bufs, sizeof(float) * 4);
    c->adam_w = (float*)dev_alloc(ctx, c->bufs, sizeof(float) * 2 * kCacheWeights);
    c->adam_t = (float*)dev_alloc(ctx, c->bufs, sizeof(float) * 4 * ne);
    c->grad_w = (float*)dev_alloc(ctx, c->bufs, sizeof(float) * kCacheWeights);
    c->grad_t = (float*)dev_alloc(ctx, c->bufs, sizeof(float) * 2 * ne);
    for (auto& b : c->bufs) if (!b.ptr) { destroy_cache_state(ctx); return set_error(ctx, S2_ERR_OOM, "cache allocation failed"); }
    if (c->bufs.size() != 9) { destroy_cache_state(ctx); return set_error(ctx, S2_ERR_OOM, "cache allocation failed"); }
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
        d.nbrick[l] = ((uint32_t)d.res[l] + 2u) / 2u;  // bricks of 2 vertices per axis over res + 1 vertices
        const double entries = 8.0 * std::pow((double)d.nbrick[l], 3.0);
        d.dense[l] = entries <= (double)(1u << c->prm.log2_table) ? 1u : 0u;
    }
    d.box_min = make_float3(c->prm.box_min[0], c->prm.box_min[1], c->prm.box_min[2]);
    d.box_inv_extent = make_float3(1.f / (c->prm.box_max[0] - c->prm.box_min[0]), 1.f / (c->prm.box_max[1] - c->prm.box_min[1]),
                                   1.f / (c->prm.box_max[2] - c->prm.box_min[2]));
    d.wimage = c->wimage;
    d.status = ctx->status_dev;
    d.grad_w = c->grad_w;
    d.grad_t = c->grad_t;
    d.loss_sum = c->loss;
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
// The inference kernel's dynamic shared memory exceeds the 48 KB default once per device.
void set_infer_attributes(S2Context* ctx) {
    static bool attr_set[64] = {};
    if (ctx->device < 64 && !attr_set[ctx->device]) {
        cudaFuncSetAttribute(k_cache_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInfSmemBytes);
        attr_set[ctx->device] = true;
    }
}

// Sets the inference kernel's attributes (once per device); callers that capture
// cache_apply_device into a CUDA graph call it first.
void cache_prepare_device(S2Context* ctx) { set_infer_attributes(ctx); }

// Path-tracer terminal vertices: accum[slot] += tput * cache(pos) for up to `cap` queries, the
// count read from n_dev.
// The device view for one inference launch: with a wait timeout armed (s2_inject_wait_timeout),
// this launch carries it and the arming is used up.
CacheDev infer_view(CacheState* c) {
    CacheDev d = c->dev;
    d.wait_test = c->inject_wait_polls;
    c->inject_wait_polls = 0;
    return d;
}

int cache_apply_device(S2Context* ctx, const float4* pos, const float4* tput, uint32_t cap, const uint32_t* n_dev,
                       float4* accum, unsigned long long* total_fx) {
    CacheState* c = ctx->cache;
    set_infer_attributes(ctx);
    const uint32_t tiles = (cap + kCacheTile - 1) / kCacheTile;
    const uint32_t grid = std::min<uint32_t>(tiles, kInfCtasPerSm * (uint32_t)c->sms);
    k_cache_infer<<<grid, kInfThreads, kInfSmemBytes, ctx->stream>>>(infer_view(c), pos, cap, n_dev, nullptr, tput, accum,
                                                                     total_fx);
    return check_cuda(ctx, cudaGetLastError(), "cache apply launch");
}

// Launches the inference kernel for n float4 positions already on the device.
int cache_infer_device(S2Context* ctx, const float4* pos, uint32_t n, float4* out) {
    CacheState* c = ctx->cache;
    if (n == 0) return S2_OK;
    set_infer_attributes(ctx);
    const uint32_t tiles = (n + kCacheTile - 1) / kCacheTile;
    const uint32_t grid = std::min<uint32_t>(tiles, kInfCtasPerSm * (uint32_t)c->sms);
    k_cache_infer<<<grid, kInfThreads, kInfSmemBytes, ctx->stream>>>(infer_view(c), pos, n, nullptr, out, nullptr, nullptr,
                                                                     nullptr);
    return check_cuda(ctx, cudaGetLastError(), "cache inference launch");
}
}  // namespace s2

extern "C" int s2_inject_wait_timeout(S2Context* ctx, uint32_t polls) {
    if (!ctx) return S2_ERR_INVALID;
    if (!ctx->cache) return set_error(ctx, S2_ERR_NO_SCENE, "s2_inject_wait_timeout before s2_cache_init");
    if (polls == 0 || polls > (1u << 20))
        return set_error(ctx, S2_ERR_INVALID, "s2_inject_wait_timeout: polls must be in 1..2^20");
    ctx->cache->inject_wait_polls = polls;
    return S2_OK;
}

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

namespace s2 {
// One forward/backward pass over n device records (n_dev: optional device count capping n);
// gradients are summed into grad_w / grad_t.
int cache_backward_device(S2Context* ctx, const float4* pos, const float4* target, uint32_t n, const uint32_t* n_dev) {
    CacheState* c = ctx->cache;
    if (n == 0) return S2_OK;
    static bool attr_set[64] = {};
    if (ctx->device < 64 && !attr_set[ctx->device]) {
        const cudaError_t e = cudaFuncSetAttribute(k_cache_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrSmemBytes);
        if (e != cudaSuccess) return check_cuda(ctx, e, "cache training kernel attributes");
        attr_set[ctx->device] = true;
    }
    const uint32_t tiles = (n + kCacheTile - 1) / kCacheTile;
    const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)c->sms);
    k_cache_train<<<grid, 128, kTrSmemBytes, ctx->stream>>>(c->dev, pos, target, n, n_dev);
    return check_cuda(ctx, cudaGetLastError(), "cache training launch");
}

// Adam step with the summed gradients of `n` records (or of *n_dev, capped at n), then the f16
// copies are refreshed.
int cache_adam_device(S2Context* ctx, uint32_t n, const uint32_t* n_dev) {
    CacheState* c = ctx->cache;
    c->step++;
    const S2CacheParams& p = c->prm;
    const float c1 = 1.f - std::pow(p.beta1, (float)c->step), c2 = 1.f - std::pow(p.beta2, (float)c->step);
    const float inv_n = 1.f / (float)std::max<uint32_t>(n, 1);
    k_cache_adam<<<(kCacheWeights + 255) / 256, 256, 0, ctx->stream>>>(c->w32, c->grad_w, c->adam_w, c->adam_w + kCacheWeights,
                                                                       kCacheWeights, inv_n, n_dev, n, p.learning_rate, p.beta1,
                                                                       p.beta2, p.epsilon, c1, c2);
    const size_t nt = 2 * (size_t)c->table_entries;
    k_cache_adam_table<<<(c->table_entries + 255) / 256, 256, 0, ctx->stream>>>(
        (float2*)c->t32, (float2*)c->grad_t, (float2*)c->adam_t, (float2*)(c->adam_t + nt), c->t16, c->table_entries, inv_n,
        n_dev, n, p.learning_rate, p.beta1, p.beta2, p.epsilon, c1, c2);
    int rc = check_cuda(ctx, cudaGetLastError(), "cache Adam launch");
    if (rc != S2_OK) return rc;
    return repack(ctx, false);  // the table's f16 copy was refreshed by the Adam pass
}
}  // namespace s2

namespace {
// host/device staging shared by s2_cache_train and s2_cache_gradients
int stage_records(S2Context* ctx, std::vector<DevBuf>& tmp, const float* positions, const float* targets, uint32_t n,
                  int on_device, const float4*& dpos, const float4*& dtgt) {
    dpos = (const float4*)positions;
    dtgt = (const float4*)targets;
    if (on_device) return S2_OK;
    dpos = (const float4*)dev_alloc(ctx, tmp, sizeof(float4) * (size_t)n);
    dtgt = (const float4*)dev_alloc(ctx, tmp, sizeof(float4) * (size_t)n);
    if (!dpos || !dtgt) return S2_ERR_OOM;
    cudaMemcpyAsync((void*)dpos, positions, sizeof(float4) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync((void*)dtgt, targets, sizeof(float4) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream);
    return S2_OK;
}

int finish(S2Context* ctx, std::vector<DevBuf>& tmp, int rc, float* loss_out, uint32_t n) {
    CacheState* c = ctx->cache;
    int status = 0;
    float loss = 0.f;
    if (rc == S2_OK) {
        cudaMemcpyAsync(&status, ctx->status_dev, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
        cudaMemcpyAsync(&loss, c->loss, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
        rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "cache training");
    }
    cudaStreamSynchronize(ctx->stream);
    free_bufs(tmp);
    if (rc == S2_OK && (status & 4)) rc = set_error(ctx, S2_ERR_TIMEOUT, "tensor-core wait timed out in cache training");
    if (rc == S2_OK && loss_out) *loss_out = loss / (float)std::max<uint32_t>(n, 1);
    return rc;
}
}  // namespace

extern "C" int s2_cache_train(S2Context* ctx, const float* positions, const float* targets, uint32_t n, float* loss,
                              int on_device) {
    if (!ctx) return S2_ERR_INVALID;
    if (!ctx->cache) return set_error(ctx, S2_ERR_NO_SCENE, "s2_cache_train before s2_cache_init");
    if (n == 0) { if (loss) *loss = 0.f; return S2_OK; }
    if (!positions || !targets) return set_error(ctx, S2_ERR_INVALID, "positions/targets is null");
    cudaSetDevice(ctx->device);
    std::vector<DevBuf> tmp;
    const float4 *dpos, *dtgt;
    int rc = stage_records(ctx, tmp, positions, targets, n, on_device, dpos, dtgt);
    if (rc != S2_OK) { free_bufs(tmp); return rc; }
    cudaMemsetAsync(ctx->status_dev, 0, sizeof(int), ctx->stream);
    cudaMemsetAsync(ctx->cache->loss, 0, sizeof(float), ctx->stream);
    rc = cache_backward_device(ctx, dpos, dtgt, n, nullptr);
    if (rc == S2_OK) rc = cache_adam_device(ctx, n, nullptr);
    return finish(ctx, tmp, rc, loss, n);
}

extern "C" int s2_cache_gradients(S2Context* ctx, const float* positions, const float* targets, uint32_t n,
                                  float* grad_weights, float* grad_table, float* loss, int on_device) {
    if (!ctx) return S2_ERR_INVALID;
    CacheState* c = ctx->cache;
    if (!c) return set_error(ctx, S2_ERR_NO_SCENE, "s2_cache_gradients before s2_cache_init");
    if (n == 0) return set_error(ctx, S2_ERR_INVALID, "s2_cache_gradients needs at least one record");
    if (!positions || !targets) return set_error(ctx, S2_ERR_INVALID, "positions/targets is null");
    cudaSetDevice(ctx->device);
    std::vector<DevBuf> tmp;
    const float4 *dpos, *dtgt;
    int rc = stage_records(ctx, tmp, positions, targets, n, on_device, dpos, dtgt);
    if (rc != S2_OK) { free_bufs(tmp); return rc; }
    const size_t nt = 2 * (size_t)c->table_entries;
    cudaMemsetAsync(c->grad_w, 0, sizeof(float) * kCacheWeights, ctx->stream);
    cudaMemsetAsync(c->grad_t, 0, sizeof(float) * nt, ctx->stream);
    cudaMemsetAsync(ctx->status_dev, 0, sizeof(int), ctx->stream);
    cudaMemsetAsync(c->loss, 0, sizeof(float), ctx->stream);
    rc = cache_backward_device(ctx, dpos, dtgt, n, nullptr);
    std::vector<float> gw(kCacheWeights), gt;
    if (rc == S2_OK) {
        cudaMemcpyAsync(gw.data(), c->grad_w, sizeof(float) * kCacheWeights, cudaMemcpyDeviceToHost, ctx->stream);
        if (grad_table) {
            gt.resize(nt);
            cudaMemcpyAsync(gt.data(), c->grad_t, sizeof(float) * nt, cudaMemcpyDeviceToHost, ctx->stream);
        }
        cudaMemsetAsync(c->grad_w, 0, sizeof(float) * kCacheWeights, ctx->stream);
        cudaMemsetAsync(c->grad_t, 0, sizeof(float) * nt, ctx->stream);
    }
    rc = finish(ctx, tmp, rc, loss, n);
    if (rc != S2_OK) return rc;
    const float inv_n = 1.f / (float)n;
    if (grad_weights) for (uint32_t i = 0; i < kCacheWeights; ++i) grad_weights[i] = gw[i] * inv_n;
    if (grad_table) for (size_t i = 0; i < nt; ++i) grad_table[i] = gt[i] * inv_n;
    return S2_OK;
}
