// C ABI: context lifecycle, scene upload, BVH build and ray queries.
//
// Replaces the reference's Scene::updateFrameData buffer uploads (src/App/Scene.cpp:428-791)
// and its hardware ray queries (src/Shaders/common/intersection.hlsli:68-338).
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "s2_context.h"
#include "s2_traverse.cuh"

using namespace s2;

namespace s2 {

int set_error(S2Context* ctx, int code, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return code;
}

int check_cuda(S2Context* ctx, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return S2_OK;
    const int code = (e == cudaErrorMemoryAllocation) ? S2_ERR_OOM : S2_ERR_CUDA;
    return set_error(ctx, code, std::string(what) + ": " + cudaGetErrorString(e));
}

void* dev_alloc(S2Context* ctx, std::vector<DevBuf>& owner, size_t bytes) {
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error(ctx, S2_ERR_OOM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
        return nullptr;
    }
    owner.push_back({p, bytes});
    return p;
}

void free_bufs(std::vector<DevBuf>& bufs) {
    for (auto& b : bufs) cudaFree(b.ptr);
    bufs.clear();
}

}  // namespace s2

#define S2_TRY(expr)                         \
    do {                                     \
        int _rc = (expr);                    \
        if (_rc != S2_OK) return _rc;        \
    } while (0)

namespace {

template <typename T>
T* upload(S2Context* ctx, std::vector<DevBuf>& owner, const T* host, size_t count) {
    T* d = (T*)dev_alloc(ctx, owner, count * sizeof(T));
    if (!d) return nullptr;
    if (count && host) {
        if (cudaMemcpyAsync(d, host, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) {
            set_error(ctx, S2_ERR_CUDA, "cudaMemcpyAsync H2D failed");
            return nullptr;
        }
    }
    return d;
}

void invert3x4(const float* m, float* out) {
    double a[3][4];
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 4; ++c) a[r][c] = m[4 * r + c];
    const double b01 = a[2][2] * a[1][1] - a[1][2] * a[2][1];
    const double b11 = -a[2][2] * a[1][0] + a[1][2] * a[2][0];
    const double b21 = a[2][1] * a[1][0] - a[1][1] * a[2][0];
    const double det = a[0][0] * b01 + a[0][1] * b11 + a[0][2] * b21;
    const double id = det != 0 ? 1.0 / det : 0.0;
    double r[3][3];
    r[0][0] = b01 * id; r[0][1] = (-a[2][2] * a[0][1] + a[0][2] * a[2][1]) * id; r[0][2] = (a[1][2] * a[0][1] - a[0][2] * a[1][1]) * id;
    r[1][0] = b11 * id; r[1][1] = (a[2][2] * a[0][0] - a[0][2] * a[2][0]) * id; r[1][2] = (-a[1][2] * a[0][0] + a[0][2] * a[1][0]) * id;
    r[2][0] = b21 * id; r[2][1] = (-a[2][1] * a[0][0] + a[0][1] * a[2][0]) * id; r[2][2] = (a[1][1] * a[0][0] - a[0][1] * a[1][0]) * id;
    for (int i = 0; i < 3; ++i) {
        const double t = -(r[i][0] * a[0][3] + r[i][1] * a[1][3] + r[i][2] * a[2][3]);
        out[4 * i + 0] = (float)r[i][0]; out[4 * i + 1] = (float)r[i][1]; out[4 * i + 2] = (float)r[i][2]; out[4 * i + 3] = (float)t;
    }
}

inline uint32_t rd_u32(const uint8_t* b, uint64_t size, uint64_t off, bool& ok) {
    if (off + 4 > size) { ok = false; return 0; }
    uint32_t v; std::memcpy(&v, b + off, 4); return v;
}
inline float rd_f32(const uint8_t* b, uint64_t size, uint64_t off, bool& ok) {
    if (off + 4 > size) { ok = false; return 0; }
    float v; std::memcpy(&v, b + off, 4); return v;
}

// Hierarchical environment-sampling tables (see DevImage): the 2x2 block probabilities that
// SampleTexel (src/Shaders/common/lights.hlsli:49-96) computes at every level of its descent, and
// the pdf SampleTexelPdf (:97-138) returns for every texel of the finest level it reaches.  Built
// only when each mip level is an exact halving of the previous one.
// Uploads `count` elements into a new scene buffer, or, for an update of an existing image (same
// dimensions, so the same sizes), over the old contents at `into`.
template <typename T>
T* put(S2Context* ctx, const T* host, size_t count, const T* into) {
    if (!into) return upload(ctx, ctx->scene_bufs, host, count);
    if (count && cudaMemcpyAsync((void*)into, host, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) {
        set_error(ctx, S2_ERR_CUDA, "cudaMemcpyAsync H2D failed");
        return nullptr;
    }
    return (T*)into;
}

void build_env_tables(S2Context* ctx, DevImage& di, const std::vector<float>& lum, const DevImage* old) {
    const uint32_t L = di.levels;
    di.nested = 0; di.quad = nullptr; di.pdf = nullptr;
    if (L < 3) return;
    for (uint32_t l = 1; l < L; ++l) {
        const bool wx = di.lw[l - 1] == 2 * di.lw[l] || (di.lw[l - 1] == 1 && di.lw[l] == 1);
        const bool hy = di.lh[l - 1] == 2 * di.lh[l] || (di.lh[l - 1] == 1 && di.lh[l] == 1);
        if (!wx || !hy) return;
    }
    const float pi = 3.14159265358979323846f;
    auto texel = [&](uint32_t l, int x, int y) -> float {
        if (x < 0 || y < 0 || x >= (int)di.lw[l] || y >= (int)di.lh[l]) return 0.f;
        return lum[di.lum_offset[l] + (size_t)y * di.lw[l] + x];
    };
    // the four luminance * sin(theta) weights of the block at (cx, cy)
    auto block = [&](uint32_t l, int cx, int cy, float p[4]) {
        const uint32_t ex = di.lw[l], ey = di.lh[l];
        const float inv_h = 1.f / (float)ey;
        p[0] = p[1] = p[2] = p[3] = 0.f;
        if ((int)ex - cx > 1) {
            const float sy = sinf(pi * (cy + 0.5f) * inv_h);
            p[0] = texel(l, cx, cy) * sy; p[1] = texel(l, cx + 1, cy) * sy;
        }
        if ((int)ey - cy > 1) {
            const float sy = sinf(pi * (cy + 1.5f) * inv_h);
            p[2] = texel(l, cx, cy + 1) * sy; p[3] = texel(l, cx + 1, cy + 1) * sy;
        }
    };
    const uint32_t lim = std::min(11u, L - 1);
    std::vector<float4> quad;
    for (uint32_t i = 1; i < lim; ++i) {
        const uint32_t l = L - 1 - i;
        const uint32_t bw = (di.lw[l] + 1) / 2, bh = (di.lh[l] + 1) / 2;
        di.quad_offset[l] = (uint32_t)quad.size();
        di.qw[l] = bw;
        for (uint32_t by = 0; by < bh; ++by) for (uint32_t bx = 0; bx < bw; ++bx) {
            float p[4];
            block(l, 2 * (int)bx, 2 * (int)by, p);
            const float sum = p[0] + p[1] + p[2] + p[3];
            if (sum < 1e-6f) quad.push_back(make_float4(-1.f, 0.f, 0.f, 0.f));
            else quad.push_back(make_float4(p[0] / sum, p[1] / sum, p[2] / sum, p[3] / sum));
        }
    }
    const uint32_t f = L - lim;  // finest level of the descent
    std::vector<float> pdf((size_t)di.lw[f] * di.lh[f]);
    for (uint32_t y = 0; y < di.lh[f]; ++y) for (uint32_t x = 0; x < di.lw[f]; ++x) {
        float pd = 1.f;
        uint32_t lx = 1, ly = 1;
        for (uint32_t i = 1; i < lim; ++i) {
            const uint32_t l = L - 1 - i;
            const int ux = (int)(x >> (l - f)), uy = (int)(y >> (l - f));
            const int cx = (ux / 2) * 2, cy = (uy / 2) * 2;
            const int ox = std::min(ux - cx, 1), oy = std::min(uy - cy, 1);
            float p[4];
            block(l, cx, cy, p);
            const float sum = p[0] + p[1] + p[2] + p[3];
            if (sum < 1e-6f) continue;
            pd *= p[oy * 2 + ox] / sum;
            lx = di.lw[l]; ly = di.lh[l];
        }
        pdf[(size_t)y * di.lw[f] + x] = pd * (float)(lx * ly);
    }
    di.quad = put(ctx, quad.data(), quad.size(), old ? old->quad : nullptr);
    di.pdf = put(ctx, pdf.data(), pdf.size(), old ? old->pdf : nullptr);
    di.pdf_level = f;
    di.nested = (di.quad && di.pdf) ? 1u : 0u;
}

// Luminance pyramid and sampling tables of the environment's bilinear footprint
// (S2_FLAG_ENV_FOOTPRINT_PDF): texel t of level 0 weighs the largest value the bilinear
// reconstruction (repeat addressing, as sample_image) takes over t's area.  The reconstruction is
// bilinear between texel centres, so that maximum is reached at a corner of one of the four
// quarter-texel rectangles: t's centre, its four edge midpoints (the mean with a neighbour) and its
// four corners (the mean of four texels).  Coarser levels average 2x2 blocks of the finer one, so
// the hierarchical descent samples a texel in proportion to its level-0 weight.
void build_env_footprint(S2Context* ctx, const DevImage& di, const std::vector<float>& lum, const DevImage* old_fp,
                         DevImage& fp) {
    fp = di;
    const int W = (int)di.lw[0], H = (int)di.lh[0];
    auto L = [&](int x, int y) {
        x %= W; if (x < 0) x += W;
        y %= H; if (y < 0) y += H;
        return lum[(size_t)y * W + x];
    };
    std::vector<float> fl;
    fl.reserve(lum.size());
    for (int y = 0; y < H; ++y) for (int x = 0; x < W; ++x) {
        const float c = L(x, y);
        float w = c;
        for (int d = -1; d <= 1; d += 2) {
            w = std::max(w, 0.5f * (c + L(x + d, y)));
            w = std::max(w, 0.5f * (c + L(x, y + d)));
            for (int e = -1; e <= 1; e += 2) w = std::max(w, 0.25f * (c + L(x + d, y) + L(x, y + e) + L(x + d, y + e)));
        }
        fl.push_back(w);
    }
    for (uint32_t l = 1; l < di.levels; ++l) {
        const uint32_t pw = di.lw[l - 1], ph = di.lh[l - 1], off = di.lum_offset[l - 1];
        for (uint32_t y = 0; y < di.lh[l]; ++y) for (uint32_t x = 0; x < di.lw[l]; ++x) {
            const uint32_t x0 = std::min(2 * x, pw - 1), x1 = std::min(2 * x + 1, pw - 1);
            const uint32_t y0 = std::min(2 * y, ph - 1), y1 = std::min(2 * y + 1, ph - 1);
            fl.push_back(0.25f * (fl[off + (size_t)y0 * pw + x0] + fl[off + (size_t)y0 * pw + x1] +
                                  fl[off + (size_t)y1 * pw + x0] + fl[off + (size_t)y1 * pw + x1]));
        }
    }
    fp.lum = put(ctx, fl.data(), fl.size(), old_fp ? old_fp->lum : nullptr);
    build_env_tables(ctx, fp, fl, old_fp);
}

// Device copy of one image (float RGBA texels); an environment image also gets its luminance mip
// pyramid and sampling tables, and in `fp` the descriptor of its footprint tables.  `old` / `old_fp`:
// the same image's current descriptors, overwritten in place.
int build_image(S2Context* ctx, uint32_t i, const S2Image& im, bool env, const DevImage* old, DevImage& di,
                const DevImage* old_fp = nullptr, DevImage* fp = nullptr) {
    if (!im.texels || im.width == 0 || im.height == 0 || im.channels < 1 || im.channels > 4)
        return set_error(ctx, S2_ERR_INVALID, "image " + std::to_string(i) + " is malformed");
    const size_t n = (size_t)im.width * im.height;
    std::vector<float> rgba(4 * n);
    for (size_t t = 0; t < n; ++t) {
        for (uint32_t c = 0; c < 4; ++c) rgba[4 * t + c] = c < im.channels ? im.texels[im.channels * t + c] : (c == 3 ? 1.f : 0.f);
    }
    di = DevImage{};
    di.width = im.width; di.height = im.height;
    di.texels = put(ctx, (const float4*)rgba.data(), n, old ? old->texels : nullptr);
    if (env) {
        // mip chain by 2x2 averaging, then luminance per texel
        std::vector<std::vector<float>> lv;
        std::vector<uint32_t> lw, lh;
        lv.push_back(rgba); lw.push_back(im.width); lh.push_back(im.height);
        while ((lw.back() > 1 || lh.back() > 1) && lv.size() < S2_MAX_IMAGE_LEVELS) {
            const uint32_t pw = lw.back(), ph = lh.back();
            const uint32_t w2 = std::max(1u, pw / 2), h2 = std::max(1u, ph / 2);
            std::vector<float> nxt(4 * (size_t)w2 * h2);
            const std::vector<float>& prev = lv.back();
            for (uint32_t y = 0; y < h2; ++y) for (uint32_t x = 0; x < w2; ++x) for (int c = 0; c < 4; ++c) {
                const uint32_t x0 = std::min(2 * x, pw - 1), x1 = std::min(2 * x + 1, pw - 1);
                const uint32_t y0 = std::min(2 * y, ph - 1), y1 = std::min(2 * y + 1, ph - 1);
                nxt[4 * ((size_t)y * w2 + x) + c] = 0.25f * (prev[4 * ((size_t)y0 * pw + x0) + c] + prev[4 * ((size_t)y0 * pw + x1) + c] +
                                                             prev[4 * ((size_t)y1 * pw + x0) + c] + prev[4 * ((size_t)y1 * pw + x1) + c]);
            }
            lv.push_back(std::move(nxt)); lw.push_back(w2); lh.push_back(h2);
        }
        std::vector<float> lum;
        di.levels = (uint32_t)lv.size();
        for (uint32_t l = 0; l < di.levels; ++l) {
            di.lum_offset[l] = (uint32_t)lum.size(); di.lw[l] = lw[l]; di.lh[l] = lh[l];
            const size_t cnt = (size_t)lw[l] * lh[l];
            for (size_t t = 0; t < cnt; ++t)
                lum.push_back(0.2126f * lv[l][4 * t] + 0.7152f * lv[l][4 * t + 1] + 0.0722f * lv[l][4 * t + 2]);
        }
        di.lum = put(ctx, lum.data(), lum.size(), old ? old->lum : nullptr);
        build_env_tables(ctx, di, lum, old);
        if (fp) build_env_footprint(ctx, di, lum, old_fp, *fp);
    }
    return S2_OK;
}

}  // namespace

// ============================================================================== lifecycle
extern "C" int s2_get_abi_version(void) { return S2_ABI_VERSION; }

extern "C" int s2_create(int device, S2Context** out) {
    if (!out) return S2_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { cudaGetLastError(); return S2_ERR_CUDA; }
    if (device < 0 || device >= n) return S2_ERR_INVALID;
    S2Context* ctx = new (std::nothrow) S2Context();
    if (!ctx) return S2_ERR_OOM;
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
        cudaMalloc(&ctx->status_dev, 64) != cudaSuccess || cudaMemset(ctx->status_dev, 0, 64) != cudaSuccess) {
        cudaGetLastError();
        s2_destroy(ctx);
        return S2_ERR_CUDA;
    }
    ctx->stream = ctx->own_stream;
    *out = ctx;
    return S2_OK;
}

extern "C" void s2_destroy(S2Context* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    destroy_render_state(ctx);
    destroy_cache_state(ctx);
    destroy_post_state(ctx);
    destroy_vcm_state(ctx);
    free_bufs(ctx->scene_bufs);
    free_bufs(ctx->bvh_bufs);
    if (ctx->status_dev) cudaFree(ctx->status_dev);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
}

extern "C" const char* s2_last_error(const S2Context* ctx) {
    if (!ctx) return "null context";
    return ctx->last_error.c_str();
}

extern "C" int s2_sync(S2Context* ctx) {
    if (!ctx) return S2_ERR_INVALID;
    cudaSetDevice(ctx->device);
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
}

extern "C" int s2_set_stream(S2Context* ctx, void* stream) {
    if (!ctx) return S2_ERR_INVALID;
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return S2_OK;
}

// ============================================================================== scene upload
extern "C" int s2_scene_upload(S2Context* ctx, const S2SceneDesc* d) {
    if (!ctx || !d) return S2_ERR_INVALID;
    cudaSetDevice(ctx->device);
    if (d->instance_count && (!d->instances || !d->transforms))
        return set_error(ctx, S2_ERR_INVALID, "instances and transforms are required");
    if (d->vertex_info_count && !d->vertex_infos) return set_error(ctx, S2_ERR_INVALID, "vertex_infos is null");
    if (d->vertex_buffer_count && (!d->vertex_buffers || !d->vertex_buffer_bytes))
        return set_error(ctx, S2_ERR_INVALID, "vertex buffers are null");
    if (d->light_count && !d->light_instance_map) return set_error(ctx, S2_ERR_INVALID, "light_instance_map is null");
    if (d->image_count && !d->images) return set_error(ctx, S2_ERR_INVALID, "images is null");
    if (d->material_bytes && !d->material_data) return set_error(ctx, S2_ERR_INVALID, "material_data is null");
    for (uint32_t i = 0; i < d->light_count; ++i)
        if (d->light_instance_map[i] >= d->instance_count) return set_error(ctx, S2_ERR_INVALID, "light_instance_map entry out of range");

    cudaStreamSynchronize(ctx->stream);
    free_bufs(ctx->scene_bufs);
    free_bufs(ctx->bvh_bufs);
    ctx->has_scene = ctx->has_bvh = false;
    destroy_render_state(ctx);
    destroy_vcm_state(ctx);  // stored reservoirs name the old scene's instances
    ctx->scene = DevScene{};
    const uint32_t ni = d->instance_count;

    // ---- flatten mesh instances to world-space triangles (host copy for the BVH build)
    ctx->tri_v0.clear(); ctx->tri_v1.clear(); ctx->tri_v2.clear(); ctx->tri_inst.clear(); ctx->tri_prim.clear();
    ctx->inst_tri_offset.assign(ni, 0);
    ctx->inst_alpha.assign(ni, 0);
    std::vector<uint32_t> prim_counts(ni, 0);
    std::vector<float> image_min_red(d->image_count, NAN);  // computed on first use
    auto min_red = [&](uint32_t k) {
        if (std::isnan(image_min_red[k])) {
            const S2Image& im = d->images[k];
            float mn = INFINITY;
            if (im.texels && im.channels >= 1)
                for (size_t t = 0; t < (size_t)im.width * im.height; ++t) mn = std::min(mn, im.texels[t * im.channels]);
            image_min_red[k] = mn;
        }
        return image_min_red[k];
    };
    for (uint32_t i = 0; i < ni; ++i) {
        const uint32_t type = d->instances[2 * i] & 0xfu;
        const uint32_t data = d->instances[2 * i + 1];
        prim_counts[i] = d->primitive_counts ? d->primitive_counts[i] : (data >> 16);
        ctx->inst_tri_offset[i] = (uint32_t)ctx->tri_inst.size();
        if (type != S2_INSTANCE_TYPE_MESH) continue;
        const uint32_t vi = data & 0xffffu;
        if (vi >= d->vertex_info_count) return set_error(ctx, S2_ERR_INVALID, "instance " + std::to_string(i) + ": vertex info index out of range");
        const uint32_t* w = d->vertex_infos + 8 * (size_t)vi;
        const uint32_t ib = w[0] & 0xffffu, pb = w[0] >> 16;
        const uint32_t istride = w[2] & 0xffu, pstride = (w[2] >> 8) & 0xffu;
        const uint32_t ioff = w[4], poff = w[5];
        if (ib >= d->vertex_buffer_count || pb >= d->vertex_buffer_count)
            return set_error(ctx, S2_ERR_INVALID, "instance " + std::to_string(i) + ": vertex buffer index out of range");
        if (istride != 2 && istride != 4) return set_error(ctx, S2_ERR_INVALID, "index stride must be 2 or 4");
        const uint8_t* ibuf = (const uint8_t*)d->vertex_buffers[ib];
        const uint8_t* pbuf = (const uint8_t*)d->vertex_buffers[pb];
        const uint64_t isz = d->vertex_buffer_bytes[ib], psz = d->vertex_buffer_bytes[pb];
        const float* m = d->transforms + 12 * (size_t)i;
        const uint32_t mat_addr = d->instances[2 * i] >> 4;
        if ((uint64_t)mat_addr + S2_MATERIAL_RECORD_BYTES > d->material_bytes)
            return set_error(ctx, S2_ERR_INVALID, "instance " + std::to_string(i) + ": material address out of range");
        {
            // non-opaque when the alpha mask has texels below the cutoff (Material::alphaTest,
            // Material.hpp:20, and the BLAS geometry flag, Scene.cpp:575)
            uint32_t mask; float cutoff;
            std::memcpy(&mask, (const uint8_t*)d->material_data + mat_addr + 48, 4);
            std::memcpy(&cutoff, (const uint8_t*)d->material_data + mat_addr + 52, 4);
            if (mask < d->image_count && !(min_red(mask) >= cutoff)) ctx->inst_alpha[i] = 1;
        }
        uint32_t max_index = 0;
        for (uint32_t p = 0; p < prim_counts[i]; ++p) {
            bool ok = true;
            uint32_t idx[3];
            const uint64_t off = (uint64_t)ioff + (uint64_t)p * 3 * istride;
            if (istride == 2) {
                for (int k = 0; k < 3; ++k) {
                    if (off + 2 * k + 2 > isz) { ok = false; break; }
                    uint16_t v; std::memcpy(&v, ibuf + off + 2 * k, 2); idx[k] = v;
                }
            } else {
                for (int k = 0; k < 3; ++k) idx[k] = rd_u32(ibuf, isz, off + 4 * k, ok);
            }
            float wv[3][3];
            for (int k = 0; k < 3 && ok; ++k) max_index = std::max(max_index, idx[k]);
            for (int k = 0; k < 3 && ok; ++k) {
                const uint64_t po = (uint64_t)poff + (uint64_t)pstride * idx[k];
                const float x = rd_f32(pbuf, psz, po, ok), y = rd_f32(pbuf, psz, po + 4, ok), z = rd_f32(pbuf, psz, po + 8, ok);
                // object -> world, evaluated left to right without contraction
                for (int r = 0; r < 3; ++r) wv[k][r] = m[4 * r + 0] * x + m[4 * r + 1] * y + m[4 * r + 2] * z + m[4 * r + 3];
            }
            if (!ok) return set_error(ctx, S2_ERR_INVALID, "instance " + std::to_string(i) + ": index or vertex read out of buffer bounds");
            for (int r = 0; r < 3; ++r) { ctx->tri_v0.push_back(wv[0][r]); ctx->tri_v1.push_back(wv[1][r]); ctx->tri_v2.push_back(wv[2][r]); }
            ctx->tri_inst.push_back(i);
            ctx->tri_prim.push_back(p);
        }
        // optional normal / texcoord streams must cover every referenced vertex
        const uint32_t nb = w[1] & 0xffffu, tb = w[1] >> 16;
        const uint64_t need_n = (uint64_t)w[6] + (uint64_t)((w[2] >> 16) & 0xffu) * max_index + 12;
        const uint64_t need_t = (uint64_t)w[7] + (uint64_t)(w[2] >> 24) * max_index + 8;
        if (prim_counts[i] && nb < d->vertex_buffer_count && need_n > d->vertex_buffer_bytes[nb])
            return set_error(ctx, S2_ERR_INVALID, "instance " + std::to_string(i) + ": normal stream out of buffer bounds");
        if (prim_counts[i] && tb < d->vertex_buffer_count && need_t > d->vertex_buffer_bytes[tb])
            return set_error(ctx, S2_ERR_INVALID, "instance " + std::to_string(i) + ": texcoord stream out of buffer bounds");
    }
    for (uint32_t l = 0; l < d->light_count; ++l) {
        const uint32_t li = d->light_instance_map[l];
        if ((d->instances[2 * li] & 0xfu) != S2_INSTANCE_TYPE_MESH || prim_counts[li] == 0)
            return set_error(ctx, S2_ERR_INVALID, "light " + std::to_string(l) + " is not a non-empty mesh instance");
    }

    // ---- device copies of the reference-format buffers
    DevScene& s = ctx->scene;
    s.instance_count = ni;
    s.instances = upload(ctx, ctx->scene_bufs, (const uint2*)d->instances, ni);
    s.prim_counts = upload(ctx, ctx->scene_bufs, prim_counts.data(), ni);
    s.transforms = upload(ctx, ctx->scene_bufs, (const float4*)d->transforms, 3 * (size_t)ni);
    std::vector<float> inv(12 * (size_t)ni), mot(12 * (size_t)ni);
    for (uint32_t i = 0; i < ni; ++i) {
        if (d->inverse_transforms) std::memcpy(&inv[12 * i], d->inverse_transforms + 12 * i, 48);
        else invert3x4(d->transforms + 12 * i, &inv[12 * i]);
        if (d->motion_transforms) std::memcpy(&mot[12 * i], d->motion_transforms + 12 * i, 48);
        else { const float id[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0}; std::memcpy(&mot[12 * i], id, 48); }
    }
    s.inv_transforms = upload(ctx, ctx->scene_bufs, (const float4*)inv.data(), 3 * (size_t)ni);
    s.motion_transforms = upload(ctx, ctx->scene_bufs, (const float4*)mot.data(), 3 * (size_t)ni);
    s.vertex_infos = upload(ctx, ctx->scene_bufs, d->vertex_infos, 8 * (size_t)d->vertex_info_count);
    std::vector<uint8_t*> vb(d->vertex_buffer_count + 1, nullptr);
    for (uint32_t i = 0; i < d->vertex_buffer_count; ++i) {
        // 16 bytes of zero padding: LoadTriangleIndices reads two aligned words for 16-bit indices
        const size_t nbytes = (size_t)d->vertex_buffer_bytes[i];
        vb[i] = (uint8_t*)dev_alloc(ctx, ctx->scene_bufs, nbytes + 16);
        if (!vb[i]) return S2_ERR_OOM;
        cudaMemsetAsync(vb[i] + nbytes, 0, 16, ctx->stream);
        if (nbytes) cudaMemcpyAsync(vb[i], d->vertex_buffers[i], nbytes, cudaMemcpyHostToDevice, ctx->stream);
    }
    ctx->vbufs_dev = upload(ctx, ctx->scene_bufs, vb.data(), vb.size());
    s.vbufs = ctx->vbufs_dev;
    s.vbuf_count = d->vertex_buffer_count;
    s.material_bytes = d->material_bytes;
    s.material_data = upload(ctx, ctx->scene_bufs, (const uint8_t*)d->material_data, d->material_bytes);
    s.light_count = d->light_count;
    s.light_instance_map = upload(ctx, ctx->scene_bufs, d->light_instance_map, d->light_count);
    std::vector<uint32_t> ilm(ni, S2_INVALID_INDEX16);
    if (d->instance_light_map) std::memcpy(ilm.data(), d->instance_light_map, 4 * (size_t)ni);
    else for (uint32_t l = 0; l < d->light_count; ++l) ilm[d->light_instance_map[l]] = l;
    s.instance_light_map = upload(ctx, ctx->scene_bufs, ilm.data(), ni);
    {
        // power-proportional pick: weight = emission luminance (material factor, textures ignored)
        // x world-space area of the light instance, floored at 1e-3 of the mean so every light
        // keeps a nonzero probability; Walker alias table (Vose's construction)
        const uint32_t L = d->light_count;
        std::vector<double> wgt(L, 0.0);
        double total = 0.0;
        for (uint32_t l = 0; l < L; ++l) {
            const uint32_t li = d->light_instance_map[l];
            const uint32_t mat = d->instances[2 * li] >> 4;
            double lum = 0.0;
            if ((size_t)mat + 36 <= d->material_bytes) {
                uint32_t w1; float esc;
                std::memcpy(&w1, (const uint8_t*)d->material_data + mat + 4, 4);
                std::memcpy(&esc, (const uint8_t*)d->material_data + mat + 32, 4);
                lum = (0.2126 * (w1 & 0xffu) + 0.7152 * ((w1 >> 8) & 0xffu) + 0.0722 * ((w1 >> 16) & 0xffu)) / 255.0 * esc;
            }
            double area = 0.0;
            for (uint32_t t = ctx->inst_tri_offset[li], e = t + prim_counts[li]; t < e && t < ctx->tri_inst.size(); ++t) {
                const float* a = &ctx->tri_v0[3 * (size_t)t]; const float* b = &ctx->tri_v1[3 * (size_t)t]; const float* c = &ctx->tri_v2[3 * (size_t)t];
                const double u[3] = {b[0] - (double)a[0], b[1] - (double)a[1], b[2] - (double)a[2]};
                const double v[3] = {c[0] - (double)a[0], c[1] - (double)a[1], c[2] - (double)a[2]};
                const double x = u[1] * v[2] - u[2] * v[1], y = u[2] * v[0] - u[0] * v[2], z = u[0] * v[1] - u[1] * v[0];
                area += 0.5 * std::sqrt(x * x + y * y + z * z);
            }
            wgt[l] = std::isfinite(lum * area) && lum * area > 0.0 ? lum * area : 0.0;
            total += wgt[l];
        }
        std::vector<float> pick(L), thr(L);
        std::vector<uint32_t> alias(L);
        if (L) {
            const double floor_w = total > 0.0 ? 1e-3 * total / L : 1.0;
            total = 0.0;
            for (uint32_t l = 0; l < L; ++l) { wgt[l] = std::max(wgt[l], floor_w); total += wgt[l]; }
            std::vector<double> q(L);
            std::vector<uint32_t> small, large;
            for (uint32_t l = 0; l < L; ++l) {
                pick[l] = (float)(wgt[l] / total);
                q[l] = wgt[l] / total * L;
                (q[l] < 1.0 ? small : large).push_back(l);
                alias[l] = l;
                thr[l] = 1.f;
            }
            while (!small.empty() && !large.empty()) {
                const uint32_t a = small.back(); small.pop_back();
                const uint32_t g = large.back();
                thr[a] = (float)q[a];
                alias[a] = g;
                q[g] -= 1.0 - q[a];
                if (q[g] < 1.0) { large.pop_back(); small.push_back(g); }
            }
            // leftovers (rounding) keep threshold 1 and alias themselves
        }
        // the sampled probability of light l is (thr[l] + sum of (1 - thr[a]) over columns a aliasing
        // to l) / L; store that exactly so pdfs match the sampling with float thresholds
        std::vector<double> eff(L, 0.0);
        for (uint32_t a = 0; a < L; ++a) { eff[a] += (double)thr[a] / L; eff[alias[a]] += (1.0 - (double)thr[a]) / L; }
        std::vector<float2> tab(std::max(1u, L));
        for (uint32_t l = 0; l < L; ++l) { uint32_t ab = alias[l]; float af; std::memcpy(&af, &ab, 4); tab[l] = make_float2(thr[l], af); pick[l] = (float)eff[l]; }
        s.light_alias = upload(ctx, ctx->scene_bufs, tab.data(), tab.size());
        if (pick.empty()) pick.push_back(0.f);
        s.light_pick_pdf = upload(ctx, ctx->scene_bufs, pick.data(), pick.size());
        s.light_power_pick = 0;
        // baked light triangles (world space, from the flattened copy): the geometric normal and
        // area follow make_shading (cross(v0 - v2, v1 - v2)), the emission LoadMaterial's 8-bit
        // colour x scale; instances with a normal stream or an emission texture are not baked
        std::vector<uint2> range(std::max(1u, L), make_uint2(0u, 0u));
        std::vector<float4> tris;
        for (uint32_t l = 0; l < L; ++l) {
            const uint32_t li = d->light_instance_map[l];
            const uint32_t mat = d->instances[2 * li] >> 4;
            const uint32_t vinfo = d->instances[2 * li + 1] & 0xffffu;
            const uint32_t nb = d->vertex_infos[8 * (size_t)vinfo + 1] & 0xffffu;
            uint32_t w1, eimg; float esc;
            std::memcpy(&w1, (const uint8_t*)d->material_data + mat + 4, 4);
            std::memcpy(&eimg, (const uint8_t*)d->material_data + mat + 20, 4);
            std::memcpy(&esc, (const uint8_t*)d->material_data + mat + 32, 4);
            const bool bake = nb >= d->vertex_buffer_count && eimg >= d->image_count;
            const float er = (float)(w1 & 0xffu) / 255.f * esc, eg = (float)((w1 >> 8) & 0xffu) / 255.f * esc,
                        eb = (float)((w1 >> 16) & 0xffu) / 255.f * esc;
            range[l] = make_uint2((uint32_t)(tris.size() / 4), prim_counts[li]);
            for (uint32_t p = 0; p < prim_counts[li]; ++p) {
                const size_t t = (size_t)ctx->inst_tri_offset[li] + p;
                const float* a = &ctx->tri_v0[3 * t]; const float* b = &ctx->tri_v1[3 * t]; const float* c = &ctx->tri_v2[3 * t];
                const float ds[3] = {a[0] - c[0], a[1] - c[1], a[2] - c[2]}, dt[3] = {b[0] - c[0], b[1] - c[1], b[2] - c[2]};
                float gn[3] = {ds[1] * dt[2] - ds[2] * dt[1], ds[2] * dt[0] - ds[0] * dt[2], ds[0] * dt[1] - ds[1] * dt[0]};
                const float area2 = std::sqrt(gn[0] * gn[0] + gn[1] * gn[1] + gn[2] * gn[2]);
                const bool ok = bake && area2 > 0.f && std::isfinite(area2);
                for (float& g : gn) g = ok ? g / area2 : 0.f;
                tris.push_back(make_float4(a[0], a[1], a[2], ok ? 0.5f * area2 : -1.f));
                tris.push_back(make_float4(b[0] - a[0], b[1] - a[1], b[2] - a[2], er));
                tris.push_back(make_float4(c[0] - a[0], c[1] - a[1], c[2] - a[2], eg));
                tris.push_back(make_float4(gn[0], gn[1], gn[2], eb));
            }
        }
        if (tris.empty()) for (int k = 0; k < 4; ++k) tris.push_back(make_float4(0.f, 0.f, 0.f, -1.f));
        s.light_tri_range = upload(ctx, ctx->scene_bufs, range.data(), range.size());
        s.light_tris = upload(ctx, ctx->scene_bufs, tris.data(), tris.size());
    }
    s.env_address = d->environment_material_address;
    if (s.env_address != S2_NO_ENVIRONMENT && (size_t)s.env_address + 16 > d->material_bytes)
        return set_error(ctx, S2_ERR_INVALID, "environment material address out of range");
    s.env_sample_prob = 0.9f;
    s.scene_sphere = make_float4(d->scene_sphere[0], d->scene_sphere[1], d->scene_sphere[2], d->scene_sphere[3]);

    // ---- images (float RGBA); the environment image also gets a luminance mip pyramid
    uint32_t env_img = S2_NO_IMAGE;
    if (s.env_address != S2_NO_ENVIRONMENT) std::memcpy(&env_img, (const uint8_t*)d->material_data + s.env_address + 12, 4);
    ctx->images_host.assign(d->image_count, DevImage{});
    ctx->env_image = -1;
    ctx->image_channels.assign(d->image_count, 0);
    ctx->env_fp_host = DevImage{};
    for (uint32_t i = 0; i < d->image_count; ++i) {
        const S2Image& im = d->images[i];
        DevImage di{};
        S2_TRY(build_image(ctx, i, im, i == env_img, nullptr, di, nullptr, &ctx->env_fp_host));
        if (i == env_img) ctx->env_image = (int)i;
        ctx->image_channels[i] = im.channels;
        ctx->images_host[i] = di;
    }
    ctx->images_dev = upload(ctx, ctx->scene_bufs, ctx->images_host.data(), ctx->images_host.size());
    s.images = ctx->images_dev;
    s.image_count = d->image_count;
    ctx->env_fp_dev = ctx->env_image >= 0 ? upload(ctx, ctx->scene_bufs, &ctx->env_fp_host, 1) : nullptr;
    s.env_fp = ctx->env_fp_dev;
    s.env_fp_on = 0;
    if (!ctx->last_error.empty() && ctx->last_error.find("cudaMalloc") != std::string::npos) return S2_ERR_OOM;
    S2_TRY(check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "scene upload"));
    ctx->has_scene = true;
    return S2_OK;
}

extern "C" int s2_update_image(S2Context* ctx, uint32_t index, const float* texels, int on_device) {
    if (!ctx) return S2_ERR_INVALID;
    if (!ctx->has_scene) return set_error(ctx, S2_ERR_NO_SCENE, "s2_update_image before s2_scene_upload");
    if (index >= ctx->images_host.size()) return set_error(ctx, S2_ERR_INVALID, "image index out of range");
    if (!texels) return set_error(ctx, S2_ERR_INVALID, "texels is null");
    cudaSetDevice(ctx->device);
    const DevImage old = ctx->images_host[index];
    S2Image im;
    im.width = old.width; im.height = old.height; im.channels = ctx->image_channels[index];
    std::vector<float> host;
    if (on_device) {
        host.resize((size_t)im.width * im.height * im.channels);
        cudaMemcpyAsync(host.data(), texels, sizeof(float) * host.size(), cudaMemcpyDeviceToHost, ctx->stream);
        S2_TRY(check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "image download"));
        im.texels = host.data();
    } else {
        im.texels = texels;
    }
    DevImage di{};
    const bool env = (int)index == ctx->env_image;
    const DevImage old_fp = ctx->env_fp_host;
    S2_TRY(build_image(ctx, index, im, env, &old, di, env ? &old_fp : nullptr, env ? &ctx->env_fp_host : nullptr));
    ctx->images_host[index] = di;
    cudaMemcpyAsync(ctx->images_dev + index, &ctx->images_host[index], sizeof(DevImage), cudaMemcpyHostToDevice, ctx->stream);
    if (env && ctx->env_fp_dev)
        cudaMemcpyAsync(ctx->env_fp_dev, &ctx->env_fp_host, sizeof(DevImage), cudaMemcpyHostToDevice, ctx->stream);
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "image update");
}

extern "C" int s2_build_bvh(S2Context* ctx, const S2BvhParams* params, S2BvhStats* stats) {
    if (!ctx) return S2_ERR_INVALID;
    if (!ctx->has_scene) return set_error(ctx, S2_ERR_NO_SCENE, "s2_build_bvh before s2_scene_upload");
    cudaSetDevice(ctx->device);
    BuildInput in;
    in.count = (uint32_t)ctx->tri_inst.size();
    in.v0 = ctx->tri_v0.data(); in.v1 = ctx->tri_v1.data(); in.v2 = ctx->tri_v2.data();
    in.instance = ctx->tri_inst.data(); in.primitive = ctx->tri_prim.data();
    BuildParams bp;
    if (params) {
        if (params->max_leaf_size) bp.max_leaf_size = params->max_leaf_size;
        if (params->sah_bins) bp.sah_bins = params->sah_bins;
        bp.threads = params->threads;
        if (params->collapse > S2_BVH_COLLAPSE_GREEDY) return set_error(ctx, S2_ERR_INVALID, "unknown BVH collapse mode");
        bp.collapse = params->collapse;
    }
    BuildOutput out;
    std::string err;
    if (build_bvh8(in, bp, out, err) != 0) return set_error(ctx, S2_ERR_INVALID, "BVH build failed: " + err);
    for (S2TriRecord& r : out.tris)
        if (ctx->inst_alpha[r.instance]) r.flat_id |= S2_TRI_ALPHA_TESTED;
    cudaStreamSynchronize(ctx->stream);
    free_bufs(ctx->bvh_bufs);
    ctx->scene.nodes = (const uint4*)upload(ctx, ctx->bvh_bufs, out.nodes.data(), out.nodes.size());
    ctx->scene.tris = (const float4*)upload(ctx, ctx->bvh_bufs, out.tris.data(), out.tris.size());
    ctx->scene.tri_count = (uint32_t)out.tris.size();
    ctx->bvh_node_count = out.nodes.size();
    if (!ctx->scene.nodes || !ctx->scene.tris) return S2_ERR_OOM;
    ctx->scene.key_lo = ctx->scene.key_scale = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!out.nodes.empty()) {  // root box: p + [0, 256) * 2^(e-127) per axis
        const S2BvhNode& root = out.nodes[0];
        const float sc[3] = {std::ldexp(256.f, (int)root.e[0] - 127), std::ldexp(256.f, (int)root.e[1] - 127),
                             std::ldexp(256.f, (int)root.e[2] - 127)};
        ctx->scene.key_lo = make_float4(root.p[0], root.p[1], root.p[2], 0.f);
        ctx->scene.key_scale = make_float4(8.f / sc[0], 8.f / sc[1], 8.f / sc[2], 0.f);
    }
    S2_TRY(bake_shading_records(ctx, ctx->bvh_bufs));
    S2_TRY(check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "BVH upload"));
    if (stats) {
        stats->node_count = out.nodes.size();
        stats->triangle_count = out.tris.size();
        stats->leaf_slot_count = out.leaf_slots;
        stats->max_depth = out.max_depth;
        stats->build_seconds = out.seconds;
        stats->sah_cost = out.sah_cost;
    }
    ctx->has_bvh = true;
    return S2_OK;
}

extern "C" int s2_get_bvh(S2Context* ctx, void* nodes, void* tris, uint64_t* counts_out) {
    if (!ctx) return S2_ERR_INVALID;
    if (!ctx->has_bvh) return set_error(ctx, S2_ERR_NO_SCENE, "s2_get_bvh before s2_build_bvh");
    if (!counts_out) return set_error(ctx, S2_ERR_INVALID, "counts_out is required");
    counts_out[0] = ctx->bvh_node_count;
    counts_out[1] = ctx->scene.tri_count;
    cudaSetDevice(ctx->device);
    if (nodes && ctx->bvh_node_count)
        cudaMemcpyAsync(nodes, ctx->scene.nodes, sizeof(S2BvhNode) * ctx->bvh_node_count, cudaMemcpyDeviceToHost, ctx->stream);
    if (tris && ctx->scene.tri_count)
        cudaMemcpyAsync(tris, ctx->scene.tris, sizeof(S2TriRecord) * (size_t)ctx->scene.tri_count, cudaMemcpyDeviceToHost,
                        ctx->stream);
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "BVH download");
}

// ============================================================================== ray queries
namespace {

constexpr int kTraceBlock = 128;

template <bool ANYHIT, bool COUNT>
__global__ void __launch_bounds__(kTraceBlock) trace_kernel(const __grid_constant__ DevScene scene,
                                                           const S2Ray* __restrict__ rays, uint32_t n, S2Hit* __restrict__ hits,
                                                           uint2* __restrict__ counts, int* __restrict__ status) {
    __shared__ uint2 stack[S2_STACK_SMEM * kTraceBlock];
    const uint32_t i = blockIdx.x * kTraceBlock + threadIdx.x;
    if (i >= n) return;
    const float4* rp = (const float4*)(rays + i);
    const float4 a = rp[0], b = rp[1];
    const TravRay r = make_trav_ray(f3(a.x, a.y, a.z), f3(b.x, b.y, b.z), a.w);
    TravHit h;
    TravCounters c{0, 0};
    const bool ok = traverse<ANYHIT, COUNT>(r, b.w, scene.nodes, scene.tris, stack + threadIdx.x, kTraceBlock, h, c,
                                            SceneAlphaTest{&scene, true});
    if (!ok) atomicOr(status, 1);
    S2Hit out;
    out.t = h.t;
    out.instance = h.instance;
    out.primitive = h.primitive;
    out.barycentrics[0] = h.b1;
    out.barycentrics[1] = h.b2;
    hits[i] = out;
    if (COUNT) counts[i] = make_uint2(c.nodes, c.tris);
}

int trace_impl(S2Context* ctx, const S2Ray* rays, uint32_t count, int anyhit, S2Hit* hits, uint32_t* fetch_counts, int on_device) {
    if (!ctx) return S2_ERR_INVALID;
    if (!ctx->has_bvh) return set_error(ctx, S2_ERR_NO_SCENE, "s2_trace before s2_build_bvh");
    if (count == 0) return S2_OK;
    if (!rays || !hits) return set_error(ctx, S2_ERR_INVALID, "rays/hits is null");
    cudaSetDevice(ctx->device);
    std::vector<DevBuf> tmp;
    const S2Ray* drays = rays;
    S2Hit* dhits = hits;
    uint2* dcounts = (uint2*)fetch_counts;
    if (!on_device) {
        drays = (const S2Ray*)dev_alloc(ctx, tmp, sizeof(S2Ray) * (size_t)count);
        dhits = (S2Hit*)dev_alloc(ctx, tmp, sizeof(S2Hit) * (size_t)count);
        dcounts = fetch_counts ? (uint2*)dev_alloc(ctx, tmp, sizeof(uint2) * (size_t)count) : nullptr;
        if (!drays || !dhits || (fetch_counts && !dcounts)) { free_bufs(tmp); return S2_ERR_OOM; }
        cudaMemcpyAsync((void*)drays, rays, sizeof(S2Ray) * (size_t)count, cudaMemcpyHostToDevice, ctx->stream);
    }
    cudaMemsetAsync(ctx->status_dev, 0, sizeof(int), ctx->stream);
    const dim3 grid((count + kTraceBlock - 1) / kTraceBlock);
    const bool counted = fetch_counts != nullptr;
    if (anyhit) {
        if (counted) trace_kernel<true, true><<<grid, kTraceBlock, 0, ctx->stream>>>(ctx->scene, drays, count, dhits, dcounts, ctx->status_dev);
        else trace_kernel<true, false><<<grid, kTraceBlock, 0, ctx->stream>>>(ctx->scene, drays, count, dhits, dcounts, ctx->status_dev);
    } else {
        if (counted) trace_kernel<false, true><<<grid, kTraceBlock, 0, ctx->stream>>>(ctx->scene, drays, count, dhits, dcounts, ctx->status_dev);
        else trace_kernel<false, false><<<grid, kTraceBlock, 0, ctx->stream>>>(ctx->scene, drays, count, dhits, dcounts, ctx->status_dev);
    }
    int rc = check_cuda(ctx, cudaGetLastError(), "trace kernel launch");
    int status = 0;
    if (rc == S2_OK) {
        if (!on_device) {
            cudaMemcpyAsync(hits, dhits, sizeof(S2Hit) * (size_t)count, cudaMemcpyDeviceToHost, ctx->stream);
            if (fetch_counts) cudaMemcpyAsync(fetch_counts, dcounts, sizeof(uint2) * (size_t)count, cudaMemcpyDeviceToHost, ctx->stream);
        }
        cudaMemcpyAsync(&status, ctx->status_dev, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
        rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "trace");
    }
    cudaStreamSynchronize(ctx->stream);
    free_bufs(tmp);
    if (rc == S2_OK && status) rc = set_error(ctx, S2_ERR_DEVICE, "traversal stack overflow");
    return rc;
}

}  // namespace

extern "C" int s2_trace(S2Context* ctx, const S2Ray* rays, uint32_t count, int anyhit, S2Hit* hits, int on_device) {
    return trace_impl(ctx, rays, count, anyhit, hits, nullptr, on_device);
}

extern "C" int s2_trace_counted(S2Context* ctx, const S2Ray* rays, uint32_t count, int anyhit, S2Hit* hits,
                                uint32_t* fetch_counts, int on_device) {
    if (!fetch_counts) return set_error(ctx, S2_ERR_INVALID, "fetch_counts is null");
    return trace_impl(ctx, rays, count, anyhit, hits, fetch_counts, on_device);
}
