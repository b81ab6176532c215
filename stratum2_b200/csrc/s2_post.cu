// Post-processing entry points: temporal accumulation of rendered frames (the Denoiser's
// temporal_accumulation pass, src/Shaders/kernels/svgf/temporal_accumulation.slang:34-129) and
// tonemapping (src/Shaders/kernels/tonemap.slang:113-192, src/App/Tonemapper.cpp:49-97).
// Both are per-pixel HBM-bound passes over the AOVs s2_render writes.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "s2_context.h"
#include "s2_math.cuh"

namespace s2 {

// History of the temporal accumulation: accumulated colour / moments (ping-pong) and the previous
// frame's visibility and depth.
struct PostState {
    std::vector<DevBuf> bufs;
    uint32_t width = 0, height = 0;
    float4* color[2] = {nullptr, nullptr};
    float2* moments[2] = {nullptr, nullptr};
    uint2* prev_vis = nullptr;
    float4* prev_depth = nullptr;
    uint32_t cur = 0;
    bool valid = false;
    unsigned int* max_buf = nullptr;  // tonemap maximum (4 x u32)
    std::vector<DevBuf> max_bufs;
    float4* filter[2] = {nullptr, nullptr};  // SVGF ping-pong images (rgb, variance)
    std::vector<DevBuf> fbufs;
    uint32_t filter_pixels = 0;
};

void destroy_post_state(S2Context* ctx) {
    if (!ctx->post) return;
    free_bufs(ctx->post->bufs);
    free_bufs(ctx->post->max_bufs);
    free_bufs(ctx->post->fbufs);
    delete ctx->post;
    ctx->post = nullptr;
}

namespace {

constexpr uint32_t kInvalidInstance16 = 0xffffu;

S2D float lum3(float3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
S2D bool bad4(float4 c) { return isnan(c.x) || isnan(c.y) || isnan(c.z) || isnan(c.w) || isinf(c.x) || isinf(c.y) || isinf(c.z) || isinf(c.w); }

struct TemporalArgs {
    int imin[2], imax[2];
    uint32_t width, height, flags, history_limit;
    float shadow_offset, shadow_scale;
    bool have_prev;
    const float4* radiance;
    const float4* albedo;
    const uint2* vis;
    const float4* depth;
    const float2* prev_uv;
    const uint2* prev_vis;
    const float4* prev_depth;
    const float4* prev_color;
    const float2* prev_moments;
    const uint32_t* instance_map;
    float4* color;
    float2* moments;
};

// temporal_accumulation.slang main (:34-129) for one pixel, debug modes left out.
__global__ void k_temporal(const __grid_constant__ TemporalArgs A) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= A.width || y >= A.height) return;
    const uint32_t ip = y * A.width + x;
    float4 color_prev = make_float4(0.f, 0.f, 0.f, 0.f);
    float2 moments_prev = make_float2(0.f, 0.f);
    float sum_w = 0.f;
    if (A.have_prev) {
        if (A.flags & S2_TEMPORAL_REPROJECT) {
            const uint2 vis = A.vis[ip];
            const float4 dep = A.depth[ip];
            const uint32_t inst = vis.x & 0xffffu;
            if (inst != kInvalidInstance16) {
                const float2 uv = A.prev_uv[ip];
                // image_min + uv * extent - 0.5; the tap origin truncates (int2()), the weights use
                // the fractional part x - floor(x), as the reference does
                const float px = (float)A.imin[0] + uv.x * (float)(A.imax[0] - A.imin[0]) - 0.5f;
                const float py = (float)A.imin[1] + uv.y * (float)(A.imax[1] - A.imin[1]) - 0.5f;
                const int p0x = (int)px, p0y = (int)py;
                const float wx = px - floorf(px), wy = py - floorf(py);
                const float3 n = unpack_normal(vis.y);
                const uint32_t mapped = A.instance_map ? A.instance_map[inst] : inst;
                // cos(degrees(2)) as written in the reference: the cosine of 114.59 radians
                const float cos_limit = cosf(2.f * 57.29577951308232f);
                const float dd = 2.f * sqrtf(dep.z * dep.z + dep.w * dep.w);
                for (int yy = 0; yy <= 1; ++yy) {
                    for (int xx = 0; xx <= 1; ++xx) {
                        const int qx = p0x + xx, qy = p0y + yy;
                        if (qx < A.imin[0] || qy < A.imin[1] || qx >= A.imax[0] || qy >= A.imax[1]) continue;
                        const uint32_t q = (uint32_t)(qy - A.imin[1]) * A.width + (uint32_t)(qx - A.imin[0]);
                        const uint2 pv = A.prev_vis[q];
                        if (mapped != (pv.x & 0xffffu)) continue;
                        if ((A.flags & S2_TEMPORAL_CHECK_NORMAL) && dot(n, unpack_normal(pv.y)) < cos_limit) continue;
                        if ((A.flags & S2_TEMPORAL_CHECK_DEPTH) && fabsf(dep.y - A.prev_depth[q].x) >= dd) continue;
                        const float4 c = A.prev_color[q];
                        if (c.w <= 0.f || bad4(c)) continue;
                        const float wc = (xx == 0 ? 1.f - wx : wx) * (yy == 0 ? 1.f - wy : wy);
                        color_prev = make_float4(color_prev.x + c.x * wc, color_prev.y + c.y * wc, color_prev.z + c.z * wc,
                                                 color_prev.w + c.w * wc);
                        const float2 m = A.prev_moments[q];
                        moments_prev = make_float2(moments_prev.x + m.x * wc, moments_prev.y + m.y * wc);
                        sum_w += wc;
                    }
                }
            }
        } else {
            color_prev = A.prev_color[ip];
            if (isnan(color_prev.x) || isnan(color_prev.y) || isnan(color_prev.z) || isinf(color_prev.x) ||
                isinf(color_prev.y) || isinf(color_prev.z))
                color_prev = make_float4(0.f, 0.f, 0.f, 0.f);
            else
                moments_prev = A.prev_moments[ip];
            sum_w = 1.f;
        }
    }
    float4 cur = A.radiance[ip];
    if ((A.flags & S2_TEMPORAL_DEMODULATE_ALBEDO) && A.albedo) {
        const float4 a = A.albedo[ip];
        cur.x /= 1e-2f + a.x; cur.y /= 1e-2f + a.y; cur.z /= 1e-2f + a.z;
    }
    if (isinf(cur.x) || isinf(cur.y) || isinf(cur.z) || cur.x != cur.x || cur.y != cur.y || cur.z != cur.z)
        cur = make_float4(0.f, 0.f, 0.f, 0.f);
    if (isinf(moments_prev.x) || isinf(moments_prev.y) || moments_prev.x != moments_prev.x || moments_prev.y != moments_prev.y)
        moments_prev = make_float2(0.f, 0.f);
    const float l = lum3(f3(cur.x, cur.y, cur.z));
    if (sum_w > 0.f && color_prev.w > 0.f) {
        const float inv = 1.f / sum_w;
        color_prev = make_float4(color_prev.x * inv, color_prev.y * inv, color_prev.z * inv, color_prev.w * inv);
        moments_prev = make_float2(moments_prev.x * inv, moments_prev.y * inv);
        float n = color_prev.w + cur.w;
        if (A.history_limit > 0 && n > (float)A.history_limit) n = (float)A.history_limit;
        float alpha = fminf(fmaxf(cur.w / n, 0.f), 1.f);
        if (A.flags & S2_TEMPORAL_SHADOW_HYSTERESIS) {
            // raise alpha where the luminance drops sharply
            const float lp = lum3(f3(color_prev.x, color_prev.y, color_prev.z));
            const float den = l + lp;
            const float r = den == 0.f ? 0.f : (lp - l) / den;
            const float s = fminf(fmaxf(r - A.shadow_offset, 0.f), 1.f);
            const float al = s * s * A.shadow_scale;
            alpha = 1.f - (1.f - alpha) * fminf(fmaxf(1.f - al, 0.f), 1.f);
        }
        A.color[ip] = make_float4(color_prev.x + (cur.x - color_prev.x) * alpha, color_prev.y + (cur.y - color_prev.y) * alpha,
                                  color_prev.z + (cur.z - color_prev.z) * alpha, n);
        A.moments[ip] = make_float2(moments_prev.x + (l - moments_prev.x) * alpha, moments_prev.y + (l * l - moments_prev.y) * alpha);
    } else {
        A.color[ip] = cur;
        A.moments[ip] = make_float2(l, l * l);
    }
}

// ---------------------------------------------------------------- SVGF
struct SvgfArgs {
    uint32_t width, height, flags, history_limit, kernel, iteration;
    int step;
    float variance_boost, sigma_boost;
    const float4* color;      // accumulated colour (rgb, history length)
    const float2* moments;
    const uint2* vis;
    const float4* depth;
    const uint32_t* instance_map;
    const float4* in;
    float4* out;
};

// estimate_variance.slang main (:26-74): temporal variance from the moments, or for short
// histories a spatial estimate over a 5x5 (7x7 for one sample) neighbourhood of the same instance.
__global__ void k_svgf_variance(const __grid_constant__ SvgfArgs A) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= (int)A.width || y >= (int)A.height) return;
    const uint32_t ip = (uint32_t)y * A.width + (uint32_t)x;
    float4 c = A.color[ip];
    float2 m = A.moments[ip];
    const uint2 vis = A.vis[ip];
    const uint32_t inst = vis.x & 0xffffu;
    const float histlen = c.w;
    if (inst == kInvalidInstance16 || histlen >= (float)A.history_limit) {
        A.out[ip] = make_float4(c.x, c.y, c.z, fabsf(m.y - m.x * m.x));
        return;
    }
    const float4 dep = A.depth[ip];
    const float3 n = unpack_normal(vis.y);
    const uint32_t mapped = A.instance_map ? A.instance_map[inst] : inst;
    float sum_w = 1.f;
    const int r = histlen > 1.f ? 2 : 3;
    for (int yy = -r; yy <= r; ++yy)
        for (int xx = -r; xx <= r; ++xx) {
            if (xx == 0 && yy == 0) continue;
            const int px = x + xx, py = y + yy;
            if (px < 0 || py < 0 || px >= (int)A.width || py >= (int)A.height) continue;
            const uint32_t q = (uint32_t)py * A.width + (uint32_t)px;
            const uint2 vp = A.vis[q];
            if (mapped != (vp.x & 0xffffu)) continue;
            const float dzl = sqrtf(dep.z * dep.z * (float)(xx * xx) + dep.w * dep.w * (float)(yy * yy));
            const float w_z = (A.flags & S2_TEMPORAL_CHECK_DEPTH) ? fabsf(A.depth[q].x - dep.x) / (dzl + 1e-2f) : 0.f;
            const float w_n = (A.flags & S2_TEMPORAL_CHECK_NORMAL) ? powf(fminf(fmaxf(dot(unpack_normal(vp.y), n), 0.f), 1.f), 128.f) : 1.f;
            const float w = expf(-w_z) * w_n;
            if (isnan(w) || isinf(w)) continue;
            const float2 mp = A.moments[q];
            const float4 cp = A.color[q];
            m = make_float2(m.x + mp.x * w, m.y + mp.y * w);
            c = make_float4(c.x + cp.x * w, c.y + cp.y * w, c.z + cp.z * w, c.w);
            sum_w += w;
        }
    const float inv = 1.f / sum_w;
    m = make_float2(m.x * inv, m.y * inv);
    c = make_float4(c.x * inv, c.y * inv, c.z * inv, c.w);
    float v = fabsf(m.y - m.x * m.x);
    if (A.variance_boost > 0.f) v *= fmaxf(1.f, A.variance_boost / (1.f + c.w));
    A.out[ip] = make_float4(c.x, c.y, c.z, v);
}

struct SvgfTap {
    float3 n_c;
    float z_c;
    float2 dz_c;
    float l_c, sigma_l;
    float4 sum;
    float sum_w;
};

// TapData::tap (atrous.slang:63-81); `off` is the offset already scaled by the step, and the depth
// term scales it by the step once more, as the shader does.
S2D void svgf_tap(const SvgfArgs& A, SvgfTap& t, int x, int y, int ox, int oy, float kw) {
    const int px = x + ox, py = y + oy;
    if (px < 0 || py < 0 || px >= (int)A.width || py >= (int)A.height) return;
    const uint32_t q = (uint32_t)py * A.width + (uint32_t)px;
    const float4 cp = A.in[q];
    const float w_l = fabsf(lum3(f3(cp.x, cp.y, cp.z)) - t.l_c) / fmaxf(t.sigma_l, 1e-10f);
    float w_z = 0.f;
    if (A.flags & S2_TEMPORAL_CHECK_DEPTH) {
        const float sx = t.dz_c.x * (float)(ox * A.step), sy = t.dz_c.y * (float)(oy * A.step);
        w_z = fabsf(A.depth[q].x - t.z_c) / (sqrtf(sx * sx + sy * sy) + 1e-2f);
    }
    const float w_n = (A.flags & S2_TEMPORAL_CHECK_NORMAL) ? powf(fmaxf(0.f, dot(unpack_normal(A.vis[q].y), t.n_c)), 256.f) : 1.f;
    const float w = expf(-w_l * w_l - w_z) * kw * w_n;
    if (isinf(w) || isnan(w)) return;
    t.sum = make_float4(t.sum.x + cp.x * w, t.sum.y + cp.y * w, t.sum.z + cp.z * w, t.sum.w + cp.w * w * w);
    t.sum_w += w;
}

// atrous.slang main (:180-227) for one iteration: edge-stopping wavelet filter of `in` into `out`.
__global__ void k_svgf_atrous(const __grid_constant__ SvgfArgs A) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= (int)A.width || y >= (int)A.height) return;
    const uint32_t ip = (uint32_t)y * A.width + (uint32_t)x;
    const uint2 vis = A.vis[ip];
    const float4 dep = A.depth[ip];
    SvgfTap t;
    t.n_c = unpack_normal(vis.y);
    t.z_c = dep.x;
    t.dz_c = make_float2(dep.z, dep.w);
    t.sum_w = 1.f;
    t.sum = A.in[ip];
    t.l_c = lum3(f3(t.sum.x, t.sum.y, t.sum.z));
    {   // compute_sigma_luminance (:48-61): the centre term is weighted by kernel[1][1] as written
        float s = t.sum.w * (1.f / 16.f);
        for (int yy = -1; yy <= 1; ++yy)
            for (int xx = -1; xx <= 1; ++xx) {
                if (xx == 0 && yy == 0) continue;
                const int px = x + xx, py = y + yy;
                if (px < 0 || py < 0 || px >= (int)A.width || py >= (int)A.height) continue;
                const float k = (xx == 0 || yy == 0) ? (1.f / 8.f) : (1.f / 16.f);
                s += A.in[(uint32_t)py * A.width + (uint32_t)px].w * k;
            }
        t.sigma_l = sqrtf(fmaxf(s, 0.f)) * A.sigma_boost;
    }
    if (!isinf(t.z_c)) {  // only foreground pixels
        const int st = A.step;
        uint32_t kernel = A.kernel;
        if (kernel == S2_SVGF_KERNEL_BOX3_SUBSAMPLED) kernel = st == 1 ? S2_SVGF_KERNEL_BOX3 : S2_SVGF_KERNEL_SUBSAMPLED;
        if (kernel == S2_SVGF_KERNEL_BOX5_SUBSAMPLED) kernel = st == 1 ? S2_SVGF_KERNEL_BOX5 : S2_SVGF_KERNEL_SUBSAMPLED;
        if (kernel == S2_SVGF_KERNEL_ATROUS) {
            // 5x5 B3-spline taps (:136-170): 2/3 at distance 1 on the axes, 1/6 at 2, products off-axis
            const float k1[3] = {1.f, 2.f / 3.f, 1.f / 6.f};
            for (int yy = -2; yy <= 2; ++yy)
                for (int xx = -2; xx <= 2; ++xx) {
                    if (xx == 0 && yy == 0) continue;
                    const int ax = xx < 0 ? -xx : xx, ay = yy < 0 ? -yy : yy;
                    const float kw = (ax == 0 || ay == 0) ? k1[ax + ay] : k1[ax] * k1[ay];
                    svgf_tap(A, t, x, y, xx * st, yy * st, kw);
                }
        } else if (kernel == S2_SVGF_KERNEL_SUBSAMPLED) {
            // (:84-118): alternating horizontal / vertical pair plus the four diagonals
            if ((A.iteration & 1u) == 0) { svgf_tap(A, t, x, y, -2 * st, 0, 1.f); svgf_tap(A, t, x, y, 2 * st, 0, 1.f); }
            else { svgf_tap(A, t, x, y, 0, -2 * st, 1.f); svgf_tap(A, t, x, y, 0, 2 * st, 1.f); }
            svgf_tap(A, t, x, y, -st, st, 1.f);
            svgf_tap(A, t, x, y, st, st, 1.f);
            svgf_tap(A, t, x, y, -st, -st, 1.f);
            svgf_tap(A, t, x, y, st, -st, 1.f);
        } else {
            const int r = kernel == S2_SVGF_KERNEL_BOX5 ? 2 : 1;  // box3 (default) / box5
            for (int yy = -r; yy <= r; ++yy)
                for (int xx = -r; xx <= r; ++xx)
                    if (xx != 0 || yy != 0) svgf_tap(A, t, x, y, xx * st, yy * st, 1.f);
        }
    }
    const float inv = 1.f / t.sum_w;
    A.out[ip] = make_float4(t.sum.x * inv, t.sum.y * inv, t.sum.z * inv, t.sum.w * inv * inv);
}

// copy_rgb (:229-236): the filtered colour of filter image 0 becomes the history's colour.
__global__ void k_svgf_copy_rgb(float4* __restrict__ color, const float4* __restrict__ filtered, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 f = filtered[i];
    color[i] = make_float4(f.x, f.y, f.z, color[i].w);
}

// ---------------------------------------------------------------- tonemapping
constexpr float kMaxQuantization = 16384.f;  // gMaxQuantization (tonemap.slang:111)

// maxReduce (tonemap.slang:113-139): per-channel and luminance maxima, quantized to 1/16384.
__global__ void k_tonemap_max(const float4* __restrict__ in, const float4* __restrict__ albedo, uint32_t n,
                              unsigned int* __restrict__ mx) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 c = in[i];
    float3 v = f3(c.x, c.y, c.z);
    if (albedo) { const float4 a = albedo[i]; v = f3(v.x * a.x, v.y * a.y, v.z * a.z); }
    const float w = lum3(v);
    if (v.x != v.x || v.y != v.y || v.z != v.z || w != w || w <= 0.f) return;
    auto q = [](float x) { return (unsigned int)fminf(fmaxf(x * kMaxQuantization, 0.f), 4294967295.f); };
    atomicMax(mx + 0, q(v.x));
    atomicMax(mx + 1, q(v.y));
    atomicMax(mx + 2, q(v.z));
    atomicMax(mx + 3, q(w));
}

S2D float3 viridis(float x) {
    // viridisQuintic (compat/common.h:96-104): a quintic fit of the viridis colour map
    const float x2 = x * x, x3 = x2 * x, x4 = x2 * x2, x5 = x4 * x;
    return f3(0.280268003f - 0.143510503f * x + 2.225793877f * x2 - 14.815088879f * x3 + 25.212752309f * x4 - 11.772589584f * x5,
              -0.002117546f + 1.617109353f * x - 1.909305070f * x2 + 2.701152864f * x3 - 1.685288385f * x4 + 0.178738871f * x5,
              0.300805501f + 2.614650302f * x - 12.019139090f * x2 + 28.933559110f * x3 - 33.491294770f * x4 + 13.762053843f * x5);
}

S2D float3 f3div(float3 a, float3 b) { return f3(a.x / b.x, a.y / b.y, a.z / b.z); }
S2D float sat(float x) { return fminf(fmaxf(x, 0.f), 1.f); }

// Uncharted 2 filmic curve (Hable), A..F as in tonemap.slang:51-71
S2D float hable(float x) {
    const float A = 0.15f, B = 0.50f, C = 0.10f, D = 0.20f, E = 0.02f, F = 0.30f;
    return ((x * (A * x + C * B) + D * E) / (x * (A * x + B) + D * F)) - E / F;
}

__global__ void k_tonemap(const float4* __restrict__ in, const float4* __restrict__ albedo, uint32_t n,
                          const unsigned int* __restrict__ mx, uint32_t mode, float scale, uint32_t flags,
                          float4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 c4 = in[i];
    float3 c = f3(c4.x, c4.y, c4.z);
    if (albedo) { const float4 a = albedo[i]; c = f3(c.x * (1e-2f + a.x), c.y * (1e-2f + a.y), c.z * (1e-2f + a.z)); }
    c = c * scale;
    const float3 maxc = f3((float)mx[0] / kMaxQuantization, (float)mx[1] / kMaxQuantization, (float)mx[2] / kMaxQuantization);
    const float maxl = (float)mx[3] / kMaxQuantization;
    switch (mode) {
    case S2_TONEMAP_REINHARD: {  // tonemap.slang:30-35
        const float l = lum3(c);
        const float3 tc = f3div(c, f3(1.f + c.x, 1.f + c.y, 1.f + c.z));
        const float3 cl = c / (1.f + l);
        c = f3(cl.x + (tc.x - cl.x) * tc.x, cl.y + (tc.y - cl.y) * tc.y, cl.z + (tc.z - cl.z) * tc.z);
        break;
    }
    case S2_TONEMAP_REINHARD_EXTENDED: {  // :36-38
        const float3 m = f3(maxc.x == 0.f ? 1.f : maxc.x, maxc.y == 0.f ? 1.f : maxc.y, maxc.z == 0.f ? 1.f : maxc.z);
        c = f3(c.x / (1.f + c.x) * (1.f + c.x / (m.x * m.x)), c.y / (1.f + c.y) * (1.f + c.y / (m.y * m.y)),
               c.z / (1.f + c.z) * (1.f + c.z / (m.z * m.z)));
        break;
    }
    case S2_TONEMAP_REINHARD_LUMINANCE: {  // :40-44
        const float l = lum3(c);
        c = c * ((l / (1.f + l)) / l);
        break;
    }
    case S2_TONEMAP_REINHARD_LUMINANCE_EXT: {  // :45-49
        const float l = lum3(c);
        const float m = maxl == 0.f ? 1.f : maxl;
        c = c * (((l / (1.f + l)) * (1.f + l / (m * m))) / l);
        break;
    }
    case S2_TONEMAP_UNCHARTED2: {  // :51-74
        const float d = hable(maxl == 0.f ? 1.f : maxl);
        c = f3(hable(c.x) / d, hable(c.y) / d, hable(c.z) / d);
        break;
    }
    case S2_TONEMAP_FILMIC: {  // :76-79 (Hejl and Burgess-Dawson)
        const float3 x = f3(fmaxf(0.f, c.x - 0.004f), fmaxf(0.f, c.y - 0.004f), fmaxf(0.f, c.z - 0.004f));
        c = f3((x.x * (6.2f * x.x + 0.5f)) / (x.x * (6.2f * x.x + 1.7f) + 0.06f),
               (x.y * (6.2f * x.y + 0.5f)) / (x.y * (6.2f * x.y + 1.7f) + 0.06f),
               (x.z * (6.2f * x.z + 0.5f)) / (x.z * (6.2f * x.z + 1.7f) + 0.06f));
        break;
    }
    case S2_TONEMAP_ACES: {  // :81-102, the fitted ACES curve of the RRT + ODT (input / output matrices)
        const float3 v = f3(0.59719f * c.x + 0.35458f * c.y + 0.04823f * c.z, 0.07600f * c.x + 0.90834f * c.y + 0.01566f * c.z,
                            0.02840f * c.x + 0.13383f * c.y + 0.83777f * c.z);
        auto fit = [](float x) { return (x * (x + 0.0245786f) - 0.000090537f) / (x * (0.983729f * x + 0.4329510f) + 0.238081f); };
        const float3 f = f3(fit(v.x), fit(v.y), fit(v.z));
        c = f3(sat(1.60475f * f.x - 0.53108f * f.y - 0.07367f * f.z), sat(-0.10208f * f.x + 1.10813f * f.y - 0.00605f * f.z),
               sat(-0.00327f * f.x - 0.07276f * f.y + 1.07602f * f.z));
        break;
    }
    case S2_TONEMAP_ACES_APPROX: {  // :104-112 (Narkowicz)
        const float3 v = c * 0.6f;
        auto ap = [](float x) { return sat((x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f)); };
        c = f3(ap(v.x), ap(v.y), ap(v.z));
        break;
    }
    case S2_TONEMAP_VIRIDIS_R:
        c = viridis(sat(lum3(c)));
        break;
    case S2_TONEMAP_VIRIDIS_LENGTH_RGB:
        c = viridis(sat(lum3(c) / (maxl == 0.f ? 1.f : maxl)));
        break;
    default:
        break;
    }
    if (flags & S2_TONEMAP_GAMMA_REFERENCE) {
        // rgbToSrgb as written in compat/common.h:88-93 (not the sRGB curve)
        auto g = [](float x) { return x <= 0.0031308f ? x * 12.92f : powf(x * 1.055f, 1.f / 2.4f) - 0.055f; };
        c = f3(g(c.x), g(c.y), g(c.z));
    } else if (flags & S2_TONEMAP_GAMMA) {
        auto g = [](float x) { return x <= 0.0031308f ? x * 12.92f : 1.055f * powf(x, 1.f / 2.4f) - 0.055f; };
        c = f3(g(c.x), g(c.y), g(c.z));
    }
    out[i] = make_float4(c.x, c.y, c.z, 1.f);
}

}  // namespace
}  // namespace s2

using namespace s2;

extern "C" void s2_default_temporal_params(S2TemporalParams* p) {
    if (!p) return;
    p->flags = S2_TEMPORAL_REPROJECT | S2_TEMPORAL_CHECK_NORMAL | S2_TEMPORAL_CHECK_DEPTH;  // Denoiser.cpp:24-26
    p->history_limit = 0;               // Denoiser.hpp:54
    p->shadow_preserve_offset = 0.1f;   // Denoiser.hpp:57
    p->shadow_preserve_scale = 1.f;     // Denoiser.hpp:58
}

extern "C" int s2_temporal_accumulate(S2Context* ctx, const S2View* view, const S2TemporalParams* prm, const S2Aovs* frame,
                                      const uint32_t* instance_index_map, float* accum_color, float* accum_moments) {
    if (!ctx) return S2_ERR_INVALID;
    if (!view || !prm || !frame || !accum_color) return set_error(ctx, S2_ERR_INVALID, "view, params, frame and accum_color are required");
    if (!frame->radiance) return set_error(ctx, S2_ERR_INVALID, "frame->radiance is required");
    const bool reproject = (prm->flags & S2_TEMPORAL_REPROJECT) != 0;
    if (reproject && (!frame->visibility || !frame->depth || !frame->prev_uv))
        return set_error(ctx, S2_ERR_INVALID, "reprojection needs the visibility, depth and prev_uv AOVs");
    if ((prm->flags & S2_TEMPORAL_DEMODULATE_ALBEDO) && !frame->albedo)
        return set_error(ctx, S2_ERR_INVALID, "albedo demodulation needs the albedo AOV");
    const int W = view->image_max[0] - view->image_min[0], H = view->image_max[1] - view->image_min[1];
    if (W <= 0 || H <= 0 || (int64_t)W * H > (1ll << 28)) return set_error(ctx, S2_ERR_INVALID, "invalid view extent");
    cudaSetDevice(ctx->device);
    if (!ctx->post) {
        ctx->post = new (std::nothrow) PostState();
        if (!ctx->post) return set_error(ctx, S2_ERR_OOM, "post-processing state allocation failed");
    }
    PostState* ps = ctx->post;
    const size_t n = (size_t)W * H;
    if (ps->width != (uint32_t)W || ps->height != (uint32_t)H) {
        free_bufs(ps->bufs);
        ps->width = ps->height = 0;
        ps->valid = false;
        for (int k = 0; k < 2; ++k) {
            ps->color[k] = (float4*)dev_alloc(ctx, ps->bufs, sizeof(float4) * n);
            ps->moments[k] = (float2*)dev_alloc(ctx, ps->bufs, sizeof(float2) * n);
        }
        ps->prev_vis = (uint2*)dev_alloc(ctx, ps->bufs, sizeof(uint2) * n);
        ps->prev_depth = (float4*)dev_alloc(ctx, ps->bufs, sizeof(float4) * n);
        for (auto& b : ps->bufs) if (!b.ptr) { free_bufs(ps->bufs); return set_error(ctx, S2_ERR_OOM, "history allocation failed"); }
        if (ps->bufs.size() != 6) { free_bufs(ps->bufs); return set_error(ctx, S2_ERR_OOM, "history allocation failed"); }
        ps->width = (uint32_t)W; ps->height = (uint32_t)H;
    }
    if (prm->flags & S2_TEMPORAL_RESET) ps->valid = false;
    TemporalArgs A;
    std::memset(&A, 0, sizeof(A));
    A.imin[0] = view->image_min[0]; A.imin[1] = view->image_min[1];
    A.imax[0] = view->image_max[0]; A.imax[1] = view->image_max[1];
    A.width = (uint32_t)W; A.height = (uint32_t)H;
    A.flags = prm->flags;
    A.history_limit = prm->history_limit;
    A.shadow_offset = prm->shadow_preserve_offset;
    A.shadow_scale = prm->shadow_preserve_scale;
    A.have_prev = ps->valid;
    A.radiance = (const float4*)frame->radiance;
    A.albedo = (const float4*)frame->albedo;
    A.vis = (const uint2*)frame->visibility;
    A.depth = (const float4*)frame->depth;
    A.prev_uv = (const float2*)frame->prev_uv;
    A.prev_vis = ps->prev_vis;
    A.prev_depth = ps->prev_depth;
    A.prev_color = ps->color[ps->cur ^ 1u];
    A.prev_moments = ps->moments[ps->cur ^ 1u];
    A.instance_map = instance_index_map;
    A.color = ps->color[ps->cur];
    A.moments = ps->moments[ps->cur];
    cudaStream_t s = ctx->stream;
    const dim3 block(16, 16), grid((W + 15) / 16, (H + 15) / 16);
    k_temporal<<<grid, block, 0, s>>>(A);
    int rc = check_cuda(ctx, cudaGetLastError(), "temporal accumulation launch");
    if (rc != S2_OK) return rc;
    cudaMemcpyAsync(accum_color, A.color, sizeof(float4) * n, cudaMemcpyDeviceToDevice, s);
    if (accum_moments) cudaMemcpyAsync(accum_moments, A.moments, sizeof(float2) * n, cudaMemcpyDeviceToDevice, s);
    // this frame's visibility and depth become the previous ones
    if (frame->visibility) cudaMemcpyAsync(ps->prev_vis, frame->visibility, sizeof(uint2) * n, cudaMemcpyDeviceToDevice, s);
    else cudaMemsetAsync(ps->prev_vis, 0xff, sizeof(uint2) * n, s);
    if (frame->depth) cudaMemcpyAsync(ps->prev_depth, frame->depth, sizeof(float4) * n, cudaMemcpyDeviceToDevice, s);
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "temporal accumulation");
    if (rc != S2_OK) return rc;
    ps->cur ^= 1u;
    ps->valid = true;
    return S2_OK;
}

extern "C" void s2_default_svgf_params(S2SvgfParams* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->iterations = 5;
    p->kernel = S2_SVGF_KERNEL_BOX3;              // Denoiser.hpp:50
    p->history_tap = 0;                           // Denoiser.hpp:49
    p->flags = S2_TEMPORAL_CHECK_NORMAL | S2_TEMPORAL_CHECK_DEPTH;
    p->history_limit = 0;
    p->variance_boost_length = 4.f;               // Denoiser.hpp:55
    p->sigma_luminance_boost = 3.f;               // Denoiser.hpp:56
}

extern "C" int s2_svgf_filter(S2Context* ctx, const S2View* view, const S2SvgfParams* prm, const S2Aovs* frame,
                              const uint32_t* instance_index_map, float* output) {
    if (!ctx) return S2_ERR_INVALID;
    if (!view || !prm || !frame || !output) return set_error(ctx, S2_ERR_INVALID, "view, params, frame and output are required");
    if (!frame->visibility || !frame->depth) return set_error(ctx, S2_ERR_INVALID, "the SVGF filter needs the visibility and depth AOVs");
    if (prm->iterations == 0 || prm->iterations > 16) return set_error(ctx, S2_ERR_INVALID, "iterations must be in 1..16");
    if (prm->kernel > S2_SVGF_KERNEL_BOX5_SUBSAMPLED) return set_error(ctx, S2_ERR_INVALID, "unknown SVGF kernel");
    const int W = view->image_max[0] - view->image_min[0], H = view->image_max[1] - view->image_min[1];
    PostState* ps = ctx->post;
    if (!ps || !ps->valid || ps->width != (uint32_t)W || ps->height != (uint32_t)H)
        return set_error(ctx, S2_ERR_INVALID, "s2_svgf_filter needs a preceding s2_temporal_accumulate of the same extent");
    cudaSetDevice(ctx->device);
    const uint32_t n = (uint32_t)W * (uint32_t)H;
    if (ps->filter_pixels != n) {
        free_bufs(ps->fbufs);
        ps->filter_pixels = 0;
        ps->filter[0] = (float4*)dev_alloc(ctx, ps->fbufs, sizeof(float4) * n);
        ps->filter[1] = (float4*)dev_alloc(ctx, ps->fbufs, sizeof(float4) * n);
        if (!ps->filter[0] || !ps->filter[1]) { free_bufs(ps->fbufs); return set_error(ctx, S2_ERR_OOM, "filter allocation failed"); }
        ps->filter_pixels = n;
    }
    const uint32_t last = ps->cur ^ 1u;  // the latest accumulation result
    SvgfArgs A;
    std::memset(&A, 0, sizeof(A));
    A.width = (uint32_t)W; A.height = (uint32_t)H;
    A.flags = prm->flags;
    A.history_limit = prm->history_limit;
    A.kernel = prm->kernel;
    A.variance_boost = prm->variance_boost_length;
    A.sigma_boost = prm->sigma_luminance_boost;
    A.color = ps->color[last];
    A.moments = ps->moments[last];
    A.vis = (const uint2*)frame->visibility;
    A.depth = (const float4*)frame->depth;
    A.instance_map = instance_index_map;
    A.out = ps->filter[0];
    cudaStream_t s = ctx->stream;
    const dim3 block(16, 16), grid((W + 15) / 16, (H + 15) / 16);
    k_svgf_variance<<<grid, block, 0, s>>>(A);
    for (uint32_t i = 0; i < prm->iterations; ++i) {
        A.iteration = i;
        A.step = 1 << i;
        A.in = ps->filter[i % 2];
        A.out = ps->filter[(i + 1) % 2];
        k_svgf_atrous<<<grid, block, 0, s>>>(A);
        if (i + 1 == prm->history_tap) k_svgf_copy_rgb<<<(n + 255) / 256, 256, 0, s>>>(ps->color[last], ps->filter[0], n);
    }
    cudaMemcpyAsync(output, ps->filter[prm->iterations % 2], sizeof(float4) * n, cudaMemcpyDeviceToDevice, s);
    int rc = check_cuda(ctx, cudaGetLastError(), "SVGF launch");
    if (rc != S2_OK) return rc;
    return check_cuda(ctx, cudaStreamSynchronize(s), "SVGF filter");
}

extern "C" int s2_tonemap(S2Context* ctx, uint32_t width, uint32_t height, const S2TonemapParams* prm, const float* input,
                          const float* albedo, float* output) {
    if (!ctx) return S2_ERR_INVALID;
    if (!prm || !input || !output) return set_error(ctx, S2_ERR_INVALID, "params, input and output are required");
    if (prm->mode > S2_TONEMAP_VIRIDIS_LENGTH_RGB) return set_error(ctx, S2_ERR_INVALID, "unknown tonemap mode");
    if (width == 0 || height == 0 || (uint64_t)width * height > (1ull << 28)) return set_error(ctx, S2_ERR_INVALID, "invalid extent");
    if (!std::isfinite(prm->exposure)) return set_error(ctx, S2_ERR_INVALID, "exposure must be finite");
    cudaSetDevice(ctx->device);
    if (!ctx->post) {
        ctx->post = new (std::nothrow) PostState();
        if (!ctx->post) return set_error(ctx, S2_ERR_OOM, "post-processing state allocation failed");
    }
    PostState* ps = ctx->post;
    if (!ps->max_buf) {
        ps->max_buf = (unsigned int*)dev_alloc(ctx, ps->max_bufs, 4 * sizeof(unsigned int));
        if (!ps->max_buf) return set_error(ctx, S2_ERR_OOM, "tonemap buffer allocation failed");
    }
    const uint32_t n = width * height;
    cudaStream_t s = ctx->stream;
    cudaMemsetAsync(ps->max_buf, 0, 4 * sizeof(unsigned int), s);  // Tonemapper.cpp:64 fillBuffer(0)
    k_tonemap_max<<<(n + 255) / 256, 256, 0, s>>>((const float4*)input, (const float4*)albedo, n, ps->max_buf);
    k_tonemap<<<(n + 255) / 256, 256, 0, s>>>((const float4*)input, (const float4*)albedo, n, ps->max_buf, prm->mode,
                                             exp2f(prm->exposure), prm->flags, (float4*)output);
    int rc = check_cuda(ctx, cudaGetLastError(), "tonemap launch");
    if (rc != S2_OK) return rc;
    return check_cuda(ctx, cudaStreamSynchronize(s), "tonemap");
}
