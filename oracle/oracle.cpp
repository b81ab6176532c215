// ORACLE -- test infrastructure only.  CPU restatement of Stratum2's path-tracing hot path,
// used by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
// The product (libstratum2_b200.so) never links, loads or calls this code.
//
// Templated on the real type: double = the FP64 correctness oracle; float = the timed FP32 CPU
// baseline and the bit-exact replica of the GPU's watertight triangle test.
//
// Parity status: the reference cannot run here (Slang shaders compiled for Vulkan, hardware ray
// queries).  Byte layouts are pinned against the reference's own compat headers
// (oracle/ref_compat.cpp, built from the reference tree when present); the shading math is pinned
// by analytic known-answer tests (furnace, irradiance, BSDF pdf normalisation, reciprocity).
// No reference-rendered golden image exists, so image parity with the reference is unpinned.
//
// Citations are paths in the Stratum2 source tree.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <vector>

#include <omp.h>

#include "../include/stratum2.h"

namespace orc {

template <class R>
struct V3 {
    R x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(R a, R b, R c) : x(a), y(b), z(c) {}
    explicit V3(R s) : x(s), y(s), z(s) {}
    R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    V3 operator+(const V3& o) const { return V3(x + o.x, y + o.y, z + o.z); }
    V3 operator-(const V3& o) const { return V3(x - o.x, y - o.y, z - o.z); }
    V3 operator*(const V3& o) const { return V3(x * o.x, y * o.y, z * o.z); }
    V3 operator/(const V3& o) const { return V3(x / o.x, y / o.y, z / o.z); }
    V3 operator*(R s) const { return V3(x * s, y * s, z * s); }
    V3 operator/(R s) const { return V3(x / s, y / s, z / s); }
    V3 operator-() const { return V3(-x, -y, -z); }
};
template <class R> V3<R> operator*(R s, const V3<R>& v) { return v * s; }
template <class R> R dot(const V3<R>& a, const V3<R>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> V3<R> cross(const V3<R>& a, const V3<R>& b) {
    return V3<R>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class R> R length(const V3<R>& a) { return std::sqrt(dot(a, a)); }
template <class R> V3<R> normalize(const V3<R>& a) { return a / std::sqrt(dot(a, a)); }
template <class R> bool any_pos(const V3<R>& a) { return a.x > 0 || a.y > 0 || a.z > 0; }
template <class R> bool all_nonpos(const V3<R>& a) { return a.x <= 0 && a.y <= 0 && a.z <= 0; }
template <class R> R luminance(const V3<R>& c) { return c.x * R(0.2126) + c.y * R(0.7152) + c.z * R(0.0722); }
template <class R> R sat(R x) { return std::min(std::max(x, R(0)), R(1)); }
template <class R> R pow2(R x) { return x * x; }
template <class R> V3<R> lerp3(const V3<R>& a, const V3<R>& b, R t) { return a + (b - a) * t; }
template <class R> R lerp1(R a, R b, R t) { return a + (b - a) * t; }
template <class R> constexpr R PI() { return R(3.14159265358979323846); }

// ------------------------------------------------------------------------------ half floats
// f32tof16/f16tof32 round trip with round-to-nearest-even (path-state fields
// testrenderer.slang:75-97 are stored as half floats).
inline float half_round(float f) {
    if (std::isnan(f)) return f;
    uint32_t u; std::memcpy(&u, &f, 4);
    const uint32_t sign = u & 0x80000000u;
    const float a = std::fabs(f);
    if (a >= 65520.f) { uint32_t r = sign | 0x7f800000u; float o; std::memcpy(&o, &r, 4); return o; }
    if (a < 6.103515625e-05f) {
        // subnormal half: quantum 2^-24
        const float q = 5.9604644775390625e-08f;
        float r = std::nearbyint(a / q) * q;
        return sign ? -r : r;
    }
    int e; std::frexp(a, &e);                 // a = m * 2^e, m in [0.5,1)
    const float q = std::ldexp(1.f, e - 11);  // 10 mantissa bits
    float r = std::nearbyint(a / q) * q;
    return sign ? -r : r;
}

// ------------------------------------------------------------------------------ RNG
// pcg4d (src/Shaders/common/rng.hlsli:23-35)
struct U4 { uint32_t x, y, z, w; };
inline U4 pcg4d(U4 v) {
    v.x = v.x * 1664525u + 1013904223u; v.y = v.y * 1664525u + 1013904223u;
    v.z = v.z * 1664525u + 1013904223u; v.w = v.w * 1664525u + 1013904223u;
    v.x += v.y * v.w; v.y += v.z * v.x; v.z += v.x * v.y; v.w += v.y * v.z;
    v.x ^= v.x >> 16; v.y ^= v.y >> 16; v.z ^= v.z >> 16; v.w ^= v.w >> 16;
    v.x += v.y * v.w; v.y += v.z * v.x; v.z += v.x * v.y; v.w += v.y * v.z;
    return v;
}
inline float u2f(uint32_t u) { uint32_t b = 0x3f800000u | (u >> 9); float f; std::memcpy(&f, &b, 4); return f - 1.f; }

// RandomSampler (rng.hlsli:39-60), and a PCG32 stream seeded from (pixel, sample)
struct Rng {
    uint32_t px, py, seed, ctr;
    bool pcg32;
    uint64_t state = 0, inc = 0;
    Rng(uint32_t x, uint32_t y, uint32_t s, bool use_pcg32) : px(x), py(y), seed(s), ctr(0), pcg32(use_pcg32) {
        if (pcg32) {
            const uint64_t initstate = ((uint64_t)s << 32) ^ 0x853c49e6748fea9bULL;
            const uint64_t initseq = ((uint64_t)y << 32) | x;
            inc = (initseq << 1u) | 1u;
            state = 0;
            step();
            state += initstate;
            step();
        }
    }
    uint32_t step() {
        const uint64_t old = state;
        state = old * 6364136223846793005ULL + (inc | 1ULL);
        const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        const uint32_t rot = (uint32_t)(old >> 59u);
        return (xs >> rot) | (xs << ((32u - rot) & 31u));
    }
    U4 next() {
        if (!pcg32) { ctr++; return pcg4d({px, py, seed, ctr}); }
        U4 r; r.x = step(); r.y = step(); r.z = step(); r.w = step(); return r;
    }
    void next_float(float out[4]) {
        U4 u = next();
        out[0] = u2f(u.x); out[1] = u2f(u.y); out[2] = u2f(u.z); out[3] = u2f(u.w);
    }
};

// ------------------------------------------------------------------------------ packing
// octahedral normal in R16G16_SNORM (common.hlsli:5-22; D3DX_DXGIFormatConvert.inl:290-330,696-713)
template <class R> int snorm16(R v) {
    if (std::isnan(v)) v = 0;
    v = std::min(std::max(v, R(-1)), R(1));
    return (int)std::trunc(v * R(32767) + (v >= 0 ? R(0.5) : R(-0.5)));
}
template <class R> uint32_t pack_normal(const V3<R>& v) {
    const R inv = R(1) / (std::fabs(v.x) + std::fabs(v.y) + std::fabs(v.z));
    R px = v.x * inv, py = v.y * inv;
    if (v.z <= 0) {
        const R ox = (R(1) - std::fabs(py)) * (px >= 0 ? R(1) : R(-1));
        const R oy = (R(1) - std::fabs(px)) * (py >= 0 ? R(1) : R(-1));
        px = ox; py = oy;
    }
    return ((uint32_t)snorm16(px) & 0xffffu) | ((uint32_t)snorm16(py) << 16);
}
template <class R> V3<R> unpack_normal(uint32_t p) {
    const int ix = (int32_t)(p << 16) >> 16, iy = (int32_t)(p & 0xffff0000u) >> 16;
    const R x = std::max(R(ix) / R(32767), R(-1)), y = std::max(R(iy) / R(32767), R(-1));
    V3<R> v(x, y, R(1) - (std::fabs(x) + std::fabs(y)));
    if (v.z < 0) {
        const R ox = (R(1) - std::fabs(v.y)) * (v.x >= 0 ? R(1) : R(-1));
        const R oy = (R(1) - std::fabs(v.x)) * (v.y >= 0 ? R(1) : R(-1));
        v.x = ox; v.y = oy;
    }
    return normalize(v);
}

// makeOrthonormal (common.hlsli:24-34)
template <class R> void make_orthonormal(const V3<R>& N, V3<R>& t, V3<R>& b) {
    if (N.x != N.y || N.x != N.z) t = V3<R>(N.z - N.y, N.x - N.z, N.y - N.x);
    else t = V3<R>(N.z - N.y, N.x + N.z, -N.y - N.x);
    t = normalize(t);
    b = cross(N, t);
}

// sampling (common.hlsli:36-76)
template <class R> void sample_concentric_disc(R u1, R u2, R& x, R& y) {
    const R ox = 2 * u1 - 1, oy = 2 * u2 - 1;
    if (ox == 0 && oy == 0) { x = y = 0; return; }
    R theta, r;
    if (std::fabs(ox) > std::fabs(oy)) { r = ox; theta = PI<R>() / 4 * (oy / ox); }
    else { r = oy; theta = PI<R>() / 2 - PI<R>() / 4 * (ox / oy); }
    x = r * std::cos(theta); y = r * std::sin(theta);
}
template <class R> V3<R> sample_cos_hemisphere(R u1, R u2) {
    R x, y; sample_concentric_disc(u1, u2, x, y);
    return V3<R>(x, y, std::sqrt(std::max(R(0), 1 - (x * x + y * y))));
}
template <class R> R cos_hemisphere_pdfw(R c) { return std::max(c, R(0)) / PI<R>(); }
template <class R> V3<R> sample_uniform_sphere(R u1, R u2) {
    const R z = u2 * 2 - 1, r = std::sqrt(std::max(1 - z * z, R(0))), phi = 2 * PI<R>() * u1;
    return V3<R>(r * std::cos(phi), r * std::sin(phi), z);
}

// rayOffset (intersection.hlsli:17-32)
template <class R> R offset_axis(R p, R n) {
    const R origin = R(1) / 32, float_scale = R(1) / 65536, int_scale = 256;
    const int of_i = (int)(int_scale * n);
    if (std::fabs(p) < origin) return p + float_scale * n;
    // the integer step is an ULP step of the float representation
    float pf = (float)p; int32_t bits; std::memcpy(&bits, &pf, 4);
    bits += (p < 0 ? -of_i : of_i);
    float r; std::memcpy(&r, &bits, 4);
    if (sizeof(R) == sizeof(float)) return (R)r;
    // FP64: the same displacement measured in float ULPs of p
    return p + ((R)r - (R)pf);
}
template <class R> V3<R> ray_offset(const V3<R>& P, V3<R> Ng, const V3<R>& dir) {
    if (dot(Ng, dir) < 0) Ng = -Ng;
    return V3<R>(offset_axis(P.x, Ng.x), offset_axis(P.y, Ng.y), offset_axis(P.z, Ng.z));
}
template <class R> R adjust_distance(R d) { return std::max(d * R(0.99), d - R(1e-2)); }

template <class R> R stable_atan2(R y, R x) {
    return x == 0 ? (y == 0 ? R(0) : (y < 0 ? -PI<R>() / 2 : PI<R>() / 2)) : std::atan2(y, x);
}
template <class R> void cart_to_uv(const V3<R>& v, R& u, R& w) {
    const R th = stable_atan2(v.z, v.x);
    u = th / PI<R>() * R(0.5) + R(0.5);
    w = std::acos(std::min(std::max(v.y, R(-1)), R(1))) / PI<R>();
}
template <class R> V3<R> uv_to_cart(R u, R v) {
    const R a = (u * 2 - 1) * PI<R>(), b = v * PI<R>();
    const R s = std::sin(b);
    return V3<R>(s * std::cos(a), std::cos(b), s * std::sin(a));
}

template <class R> R mis(R a, R b) {
    if (std::isinf(a)) return std::isinf(b) ? R(0.5) : R(1);
    const R a2 = a * a;
    return a2 / (a2 + b * b);
}

// ------------------------------------------------------------------------------ scene
struct Tri { uint32_t inst, prim; };

template <class R>
struct Image {
    uint32_t w = 0, h = 0;
    std::vector<float> rgba;
    // luminance pyramid (environment only)
    std::vector<std::vector<R>> lum;
    std::vector<uint32_t> lw, lh;
    V3<R> sample(R u, R v, R* alpha = nullptr) const {
        const R x = u * w - R(0.5), y = v * h - R(0.5);
        const R fx = std::floor(x), fy = std::floor(y);
        const R ax = x - fx, ay = y - fy;
        int x0 = (int)fx % (int)w; if (x0 < 0) x0 += w;
        int y0 = (int)fy % (int)h; if (y0 < 0) y0 += h;
        const int x1 = (x0 + 1) % (int)w, y1 = (y0 + 1) % (int)h;
        auto T = [&](int xx, int yy, int c) { return (R)rgba[4 * ((size_t)yy * w + xx) + c]; };
        V3<R> r;
        R out[4];
        for (int c = 0; c < 4; ++c)
            out[c] = T(x0, y0, c) * (1 - ax) * (1 - ay) + T(x1, y0, c) * ax * (1 - ay) + T(x0, y1, c) * (1 - ax) * ay + T(x1, y1, c) * ax * ay;
        if (alpha) *alpha = out[3];
        return V3<R>(out[0], out[1], out[2]);
    }
};

struct BNode { double lo[3], hi[3]; int32_t left, right; uint32_t begin, count; };

template <class R>
struct Scene {
    uint32_t ni = 0;
    std::vector<uint32_t> inst_word0, inst_word1, prim_count;
    std::vector<R> xf, inv, motion;  // 12 per instance
    std::vector<uint32_t> vinfo;     // 8 per
    std::vector<std::vector<uint8_t>> vbuf;
    std::vector<uint8_t> mat;
    std::vector<uint32_t> light_map, inst_light_map;
    uint32_t env_addr = S2_NO_ENVIRONMENT;
    std::vector<Image<R>> images;
    Image<R> env_fp;  // the environment image with its bilinear-footprint luminance pyramid
    int env_image = -1;
    R sphere[4];
    // flattened triangles + BVH2
    std::vector<R> tv;               // 9 per triangle
    std::vector<Tri> tid;
    std::vector<BNode> nodes;
    std::vector<uint32_t> order;
    bool exact32 = false;            // triangles flattened with the GPU's float expression

    uint32_t u32(const std::vector<uint8_t>& b, size_t off) const { uint32_t v; std::memcpy(&v, b.data() + off, 4); return v; }
    float f32(const std::vector<uint8_t>& b, size_t off) const { float v; std::memcpy(&v, b.data() + off, 4); return v; }

    V3<R> xpoint(const R* m, const V3<R>& p) const {
        return V3<R>(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3], m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
                     m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]);
    }
    V3<R> xvec(const R* m, const V3<R>& v) const {
        return V3<R>(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[4] * v.x + m[5] * v.y + m[6] * v.z, m[8] * v.x + m[9] * v.y + m[10] * v.z);
    }

    // LoadTriangleIndices (scene.hlsli:43-62)
    void tri_indices(uint32_t inst, uint32_t prim, uint32_t idx[3]) const {
        const uint32_t* w = &vinfo[8 * (size_t)(inst_word1[inst] & 0xffffu)];
        const uint32_t ib = w[0] & 0xffffu, stride = w[2] & 0xffu, off = w[4];
        const std::vector<uint8_t>& b = vbuf[ib];
        const size_t o = (size_t)off + (size_t)prim * 3 * stride;
        for (int k = 0; k < 3; ++k) {
            if (stride == 2) { uint16_t v; std::memcpy(&v, b.data() + o + 2 * k, 2); idx[k] = v; }
            else idx[k] = u32(b, o + 4 * k);
        }
    }
    V3<R> position(uint32_t inst, uint32_t vi) const {
        const uint32_t* w = &vinfo[8 * (size_t)(inst_word1[inst] & 0xffffu)];
        const uint32_t pb = w[0] >> 16, stride = (w[2] >> 8) & 0xffu, off = w[5];
        const size_t o = (size_t)off + (size_t)stride * vi;
        return V3<R>(f32(vbuf[pb], o), f32(vbuf[pb], o + 4), f32(vbuf[pb], o + 8));
    }
    bool attr2(uint32_t inst, uint32_t vi, R out[2]) const {
        const uint32_t* w = &vinfo[8 * (size_t)(inst_word1[inst] & 0xffffu)];
        const uint32_t tb = w[1] >> 16, stride = w[2] >> 24, off = w[7];
        if (tb >= vbuf.size()) return false;
        const size_t o = (size_t)off + (size_t)stride * vi;
        out[0] = f32(vbuf[tb], o); out[1] = f32(vbuf[tb], o + 4);
        return true;
    }
    bool attr_normal(uint32_t inst, uint32_t vi, V3<R>& n) const {
        const uint32_t* w = &vinfo[8 * (size_t)(inst_word1[inst] & 0xffffu)];
        const uint32_t nb = w[1] & 0xffffu, stride = (w[2] >> 16) & 0xffu, off = w[6];
        if (nb >= vbuf.size()) return false;
        const size_t o = (size_t)off + (size_t)stride * vi;
        n = V3<R>(f32(vbuf[nb], o), f32(vbuf[nb], o + 4), f32(vbuf[nb], o + 8));
        return true;
    }

    bool load(const S2SceneDesc* d, bool exact_float) {
        exact32 = exact_float;
        ni = d->instance_count;
        inst_word0.resize(ni); inst_word1.resize(ni); prim_count.resize(ni);
        xf.resize(12 * (size_t)ni); inv.resize(12 * (size_t)ni); motion.resize(12 * (size_t)ni);
        for (uint32_t i = 0; i < ni; ++i) {
            inst_word0[i] = d->instances[2 * i]; inst_word1[i] = d->instances[2 * i + 1];
            prim_count[i] = d->primitive_counts ? d->primitive_counts[i] : (inst_word1[i] >> 16);
            for (int k = 0; k < 12; ++k) xf[12 * i + k] = (R)d->transforms[12 * i + k];
            // inverse in the working precision
            const R* m = &xf[12 * i];
            const R b01 = m[10] * m[5] - m[6] * m[9], b11 = -m[10] * m[4] + m[6] * m[8], b21 = m[9] * m[4] - m[5] * m[8];
            const R det = m[0] * b01 + m[1] * b11 + m[2] * b21, id = R(1) / det;
            R r[9] = {b01 * id, (-m[10] * m[1] + m[2] * m[9]) * id, (m[6] * m[1] - m[2] * m[5]) * id,
                      b11 * id, (m[10] * m[0] - m[2] * m[8]) * id, (-m[6] * m[0] + m[2] * m[4]) * id,
                      b21 * id, (-m[9] * m[0] + m[1] * m[8]) * id, (m[5] * m[0] - m[1] * m[4]) * id};
            for (int row = 0; row < 3; ++row) {
                inv[12 * i + 4 * row + 0] = r[3 * row]; inv[12 * i + 4 * row + 1] = r[3 * row + 1]; inv[12 * i + 4 * row + 2] = r[3 * row + 2];
                inv[12 * i + 4 * row + 3] = -(r[3 * row] * m[3] + r[3 * row + 1] * m[7] + r[3 * row + 2] * m[11]);
            }
            if (d->inverse_transforms) for (int k = 0; k < 12; ++k) inv[12 * i + k] = (R)d->inverse_transforms[12 * i + k];
            for (int k = 0; k < 12; ++k) motion[12 * i + k] = d->motion_transforms ? (R)d->motion_transforms[12 * i + k] : (R)((k % 5) == 0 ? 1 : 0);
        }
        vinfo.assign(d->vertex_infos, d->vertex_infos + 8 * (size_t)d->vertex_info_count);
        vbuf.resize(d->vertex_buffer_count);
        for (uint32_t i = 0; i < d->vertex_buffer_count; ++i) {
            const uint8_t* p = (const uint8_t*)d->vertex_buffers[i];
            vbuf[i].assign(p, p + d->vertex_buffer_bytes[i]);
            vbuf[i].resize(vbuf[i].size() + 8, 0);  // tail padding for the 16-bit index double-word read
        }
        mat.assign((const uint8_t*)d->material_data, (const uint8_t*)d->material_data + d->material_bytes);
        mat.resize(mat.size() + 64, 0);
        light_map.assign(d->light_instance_map, d->light_instance_map + d->light_count);
        inst_light_map.assign(ni, S2_INVALID_INDEX16);
        for (uint32_t l = 0; l < d->light_count; ++l) inst_light_map[light_map[l]] = l;
        env_addr = d->environment_material_address;
        for (int k = 0; k < 4; ++k) sphere[k] = (R)d->scene_sphere[k];
        uint32_t env_img = S2_NO_IMAGE;
        if (env_addr != S2_NO_ENVIRONMENT) env_img = u32(mat, env_addr + 12);
        images.resize(d->image_count);
        for (uint32_t i = 0; i < d->image_count; ++i) {
            const S2Image& im = d->images[i];
            Image<R>& o = images[i];
            o.w = im.width; o.h = im.height;
            const size_t n = (size_t)im.width * im.height;
            o.rgba.resize(4 * n);
            for (size_t t = 0; t < n; ++t)
                for (uint32_t c = 0; c < 4; ++c) o.rgba[4 * t + c] = c < im.channels ? im.texels[im.channels * t + c] : (c == 3 ? 1.f : 0.f);
            if (i == env_img) {
                // mip chain of 2x2 averages, then luminance (the GPU builds the same pyramid)
                std::vector<std::vector<R>> lv(1);
                lv[0].resize(4 * n);
                for (size_t t = 0; t < 4 * n; ++t) lv[0][t] = (R)o.rgba[t];
                o.lw.push_back(o.w); o.lh.push_back(o.h);
                while ((o.lw.back() > 1 || o.lh.back() > 1) && lv.size() < 16) {
                    const uint32_t pw = o.lw.back(), ph = o.lh.back();
                    const uint32_t w2 = std::max(1u, pw / 2), h2 = std::max(1u, ph / 2);
                    std::vector<R> nx(4 * (size_t)w2 * h2);
                    const std::vector<R>& pv = lv.back();
                    for (uint32_t y = 0; y < h2; ++y) for (uint32_t x = 0; x < w2; ++x) for (int c = 0; c < 4; ++c) {
                        const uint32_t x0 = std::min(2 * x, pw - 1), x1 = std::min(2 * x + 1, pw - 1);
                        const uint32_t y0 = std::min(2 * y, ph - 1), y1 = std::min(2 * y + 1, ph - 1);
                        nx[4 * ((size_t)y * w2 + x) + c] = R(0.25) * (pv[4 * ((size_t)y0 * pw + x0) + c] + pv[4 * ((size_t)y0 * pw + x1) + c] +
                                                                      pv[4 * ((size_t)y1 * pw + x0) + c] + pv[4 * ((size_t)y1 * pw + x1) + c]);
                    }
                    lv.push_back(std::move(nx)); o.lw.push_back(w2); o.lh.push_back(h2);
                }
                o.lum.resize(lv.size());
                for (size_t l = 0; l < lv.size(); ++l) {
                    const size_t cnt = lv[l].size() / 4;
                    o.lum[l].resize(cnt);
                    for (size_t t = 0; t < cnt; ++t)
                        o.lum[l][t] = R(0.2126) * lv[l][4 * t] + R(0.7152) * lv[l][4 * t + 1] + R(0.0722) * lv[l][4 * t + 2];
                }
                env_image = (int)i;
                // S2_FLAG_ENV_FOOTPRINT_PDF: level 0 weighs the largest value of the bilinear
                // luminance over each texel's area (its centre, edge midpoints and corners, repeat
                // addressing); coarser levels average 2x2 blocks
                env_fp = o;
                const int W = (int)o.lw[0], H = (int)o.lh[0];
                auto L = [&](int x, int y) {
                    x %= W; if (x < 0) x += W;
                    y %= H; if (y < 0) y += H;
                    return o.lum[0][(size_t)y * W + x];
                };
                for (int y = 0; y < H; ++y) for (int x = 0; x < W; ++x) {
                    const R c = L(x, y);
                    R w = c;
                    for (int dd = -1; dd <= 1; dd += 2) {
                        w = std::max(w, R(0.5) * (c + L(x + dd, y)));
                        w = std::max(w, R(0.5) * (c + L(x, y + dd)));
                        for (int e = -1; e <= 1; e += 2) w = std::max(w, R(0.25) * (c + L(x + dd, y) + L(x, y + e) + L(x + dd, y + e)));
                    }
                    env_fp.lum[0][(size_t)y * W + x] = w;
                }
                for (size_t l = 1; l < env_fp.lum.size(); ++l) {
                    const uint32_t pw = o.lw[l - 1], ph = o.lh[l - 1];
                    for (uint32_t y = 0; y < o.lh[l]; ++y) for (uint32_t x = 0; x < o.lw[l]; ++x) {
                        const uint32_t x0 = std::min(2 * x, pw - 1), x1 = std::min(2 * x + 1, pw - 1);
                        const uint32_t y0 = std::min(2 * y, ph - 1), y1 = std::min(2 * y + 1, ph - 1);
                        const std::vector<R>& f = env_fp.lum[l - 1];
                        env_fp.lum[l][(size_t)y * o.lw[l] + x] = R(0.25) * (f[(size_t)y0 * pw + x0] + f[(size_t)y0 * pw + x1] +
                                                                            f[(size_t)y1 * pw + x0] + f[(size_t)y1 * pw + x1]);
                    }
                }
            }
        }
        // flatten triangles
        tv.clear(); tid.clear();
        for (uint32_t i = 0; i < ni; ++i) {
            if ((inst_word0[i] & 0xfu) != S2_INSTANCE_TYPE_MESH) continue;
            const float* mf = d->transforms + 12 * (size_t)i;
            for (uint32_t p = 0; p < prim_count[i]; ++p) {
                uint32_t idx[3]; tri_indices(i, p, idx);
                for (int k = 0; k < 3; ++k) {
                    const V3<R> v = position(i, idx[k]);
                    if (exact32) {
                        const float x = (float)v.x, y = (float)v.y, z = (float)v.z;
                        for (int r = 0; r < 3; ++r) tv.push_back((R)(mf[4 * r] * x + mf[4 * r + 1] * y + mf[4 * r + 2] * z + mf[4 * r + 3]));
                    } else {
                        const V3<R> w = xpoint(&xf[12 * i], v);
                        tv.push_back(w.x); tv.push_back(w.y); tv.push_back(w.z);
                    }
                }
                tid.push_back({i, p});
            }
        }
        build_bvh();
        return true;
    }

    // ---- BVH2: median split on the longest centroid axis, boxes in double padded outward
    void build_bvh() {
        const uint32_t n = (uint32_t)tid.size();
        order.resize(n);
        for (uint32_t i = 0; i < n; ++i) order[i] = i;
        nodes.clear();
        nodes.reserve(2 * (size_t)n + 1);
        std::vector<double> cen(3 * (size_t)n);
        for (uint32_t i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) cen[3 * i + k] = ((double)tv[9 * i + k] + (double)tv[9 * i + 3 + k] + (double)tv[9 * i + 6 + k]) / 3;
        nodes.push_back(BNode{});
        struct Job { uint32_t node, begin, count; };
        std::vector<Job> st{{0, 0, n}};
        while (!st.empty()) {
            Job j = st.back(); st.pop_back();
            BNode nd{};
            nd.left = nd.right = -1; nd.begin = j.begin; nd.count = j.count;
            double clo[3] = {1e300, 1e300, 1e300}, chi[3] = {-1e300, -1e300, -1e300};
            for (int k = 0; k < 3; ++k) { nd.lo[k] = 1e300; nd.hi[k] = -1e300; }
            for (uint32_t q = j.begin; q < j.begin + j.count; ++q) {
                const uint32_t t = order[q];
                for (int v = 0; v < 3; ++v) for (int k = 0; k < 3; ++k) {
                    nd.lo[k] = std::min(nd.lo[k], (double)tv[9 * t + 3 * v + k]);
                    nd.hi[k] = std::max(nd.hi[k], (double)tv[9 * t + 3 * v + k]);
                }
                for (int k = 0; k < 3; ++k) { clo[k] = std::min(clo[k], cen[3 * t + k]); chi[k] = std::max(chi[k], cen[3 * t + k]); }
            }
            for (int k = 0; k < 3; ++k) {
                const double pad = 1e-5 * (std::fabs(nd.lo[k]) + std::fabs(nd.hi[k]) + (nd.hi[k] - nd.lo[k])) + 1e-9;
                nd.lo[k] -= pad; nd.hi[k] += pad;
            }
            if (j.count > 4) {
                int ax = 0;
                for (int k = 1; k < 3; ++k) if (chi[k] - clo[k] > chi[ax] - clo[ax]) ax = k;
                const uint32_t mid = j.begin + j.count / 2;
                std::nth_element(order.begin() + j.begin, order.begin() + mid, order.begin() + j.begin + j.count,
                                 [&](uint32_t a, uint32_t b) { return cen[3 * a + ax] < cen[3 * b + ax]; });
                nd.left = (int32_t)nodes.size(); nodes.push_back(BNode{});
                nd.right = (int32_t)nodes.size(); nodes.push_back(BNode{});
                st.push_back({(uint32_t)nd.left, j.begin, mid - j.begin});
                st.push_back({(uint32_t)nd.right, mid, j.begin + j.count - mid});
            }
            nodes[j.node] = nd;
        }
    }
};

// ------------------------------------------------------------------------------ ray/triangle
// Watertight test (Woop, Benthin, Wald 2013); the float version evaluates exactly the GPU's
// operation sequence (no contraction: this file is compiled with -ffp-contract=off).
template <class R> struct WRay {
    V3<R> o, d; R tmin;
    int kx, ky, kz; R Sx, Sy, Sz;
    double inv[3];
};
template <class R> WRay<R> make_wray(const V3<R>& o, const V3<R>& d, R tmin) {
    WRay<R> r; r.o = o; r.d = d; r.tmin = tmin;
    const R ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
    int kz = (ax > ay) ? ((ax > az) ? 0 : 2) : ((ay > az) ? 1 : 2);
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    if (d[kz] < 0) std::swap(kx, ky);
    r.kx = kx; r.ky = ky; r.kz = kz;
    r.Sx = d[kx] / d[kz]; r.Sy = d[ky] / d[kz]; r.Sz = R(1) / d[kz];
    for (int k = 0; k < 3; ++k) { double dk = (double)d[k]; if (std::fabs(dk) < 1e-300) dk = std::copysign(1e-300, dk); r.inv[k] = 1.0 / dk; }
    return r;
}
template <class R> bool isect_tri(const WRay<R>& r, const R* v, R tmax, R& t_out, R& b1, R& b2) {
    const V3<R> A = V3<R>(v[0], v[1], v[2]) - r.o, B = V3<R>(v[3], v[4], v[5]) - r.o, C = V3<R>(v[6], v[7], v[8]) - r.o;
    const R Ax = A[r.kx] - r.Sx * A[r.kz], Ay = A[r.ky] - r.Sy * A[r.kz];
    const R Bx = B[r.kx] - r.Sx * B[r.kz], By = B[r.ky] - r.Sy * B[r.kz];
    const R Cx = C[r.kx] - r.Sx * C[r.kz], Cy = C[r.ky] - r.Sy * C[r.kz];
    R U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
    if (U == 0 || V == 0 || W == 0) {
        if (sizeof(R) == sizeof(float)) {
            U = (R)((double)Cx * (double)By - (double)Cy * (double)Bx);
            V = (R)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
            W = (R)((double)Bx * (double)Ay - (double)By * (double)Ax);
        } else {
            U = (R)((long double)Cx * By - (long double)Cy * Bx);
            V = (R)((long double)Ax * Cy - (long double)Ay * Cx);
            W = (R)((long double)Bx * Ay - (long double)By * Ax);
        }
    }
    if ((U < 0 || V < 0 || W < 0) && (U > 0 || V > 0 || W > 0)) return false;
    const R det = U + V + W;
    if (det == 0) return false;
    const R Az = r.Sz * A[r.kz], Bz = r.Sz * B[r.kz], Cz = r.Sz * C[r.kz];
    const R T = U * Az + V * Bz + W * Cz;
    const R t = T / det;
    if (!(t >= r.tmin && t <= tmax)) return false;
    t_out = t; b1 = V / det; b2 = W / det;
    return true;
}

template <class R> struct Hit { R t; uint32_t tri; R b1, b2; bool hit; };

// Candidate test of a non-opaque triangle (intersection.hlsli:125-146): the alpha-mask image of
// the instance's material (index and cutoff at bytes 48/52, material.hlsli:72-76) at the hit's
// texture coordinate, level 0, red channel, >= cutoff.  Materials without a mask always pass.
template <class R> bool alpha_pass(const Scene<R>& s, uint32_t inst, uint32_t prim, R b1, R b2) {
    const uint32_t mat = s.inst_word0[inst] >> 4;
    const uint32_t mask = s.u32(s.mat, mat + 48);
    if (mask >= s.images.size()) return true;
    const float cutoff = s.f32(s.mat, mat + 52);
    uint32_t idx[3]; s.tri_indices(inst, prim, idx);
    R t0[2] = {0, 0}, t1[2] = {0, 0}, t2[2] = {0, 0};
    if (s.attr2(inst, idx[0], t0)) { s.attr2(inst, idx[1], t1); s.attr2(inst, idx[2], t2); }
    const R u = t0[0] + (t1[0] - t0[0]) * b1 + (t2[0] - t0[0]) * b2;
    const R v = t0[1] + (t1[1] - t0[1]) * b1 + (t2[1] - t0[1]) * b2;
    return s.images[mask].sample(u, v).x >= (R)cutoff;
}

template <class R> Hit<R> trace(const Scene<R>& s, const V3<R>& o, const V3<R>& d, R tmin, R tmax, bool anyhit,
                                bool alpha_test = true) {
    Hit<R> h{tmax, 0xffffffffu, 0, 0, false};
    if (s.nodes.empty() || s.tid.empty()) return h;
    const WRay<R> r = make_wray(o, d, tmin);
    const double od[3] = {(double)o.x, (double)o.y, (double)o.z};
    uint32_t stack[256]; int sp = 0;
    stack[sp++] = 0;
    uint32_t best_inst = 0xffffffffu, best_prim = 0xffffffffu;
    while (sp) {
        const BNode& n = s.nodes[stack[--sp]];
        double t0 = (double)tmin, t1 = (double)h.t;
        bool miss = false;
        for (int k = 0; k < 3 && !miss; ++k) {
            double a = (n.lo[k] - od[k]) * r.inv[k], b = (n.hi[k] - od[k]) * r.inv[k];
            if (a > b) std::swap(a, b);
            if (std::isnan(a) || std::isnan(b)) continue;
            t0 = std::max(t0, a); t1 = std::min(t1, b * (1 + 1e-9));
            if (t0 > t1 * (1 + 1e-9) + 1e-12) miss = true;
        }
        if (miss) continue;
        if (n.left < 0) {
            for (uint32_t q = n.begin; q < n.begin + n.count; ++q) {
                const uint32_t ti = s.order[q];
                R t, b1, b2;
                if (isect_tri(r, &s.tv[9 * (size_t)ti], h.t, t, b1, b2)) {
                    const uint32_t inst = s.tid[ti].inst, prim = s.tid[ti].prim;
                    if (alpha_test && !alpha_pass(s, inst, prim, b1, b2)) continue;
                    if (anyhit) { h.t = t; h.tri = ti; h.b1 = b1; h.b2 = b2; h.hit = true; return h; }
                    if (t < h.t || inst < best_inst || (inst == best_inst && prim < best_prim)) {
                        h.t = t; h.tri = ti; h.b1 = b1; h.b2 = b2; h.hit = true; best_inst = inst; best_prim = prim;
                    }
                }
            }
        } else {
            // push the far child first
            const BNode& L = s.nodes[n.left];
            const BNode& Rn = s.nodes[n.right];
            double cl = 0, cr = 0;
            for (int k = 0; k < 3; ++k) { cl += ((L.lo[k] + L.hi[k]) * 0.5 - od[k]) * (double)d[k]; cr += ((Rn.lo[k] + Rn.hi[k]) * 0.5 - od[k]) * (double)d[k]; }
            if (sp + 2 > 256) return h;
            if (cl < cr) { stack[sp++] = n.right; stack[sp++] = n.left; }
            else { stack[sp++] = n.left; stack[sp++] = n.right; }
        }
    }
    return h;
}

}  // namespace orc

#include "oracle_pt.inl"

// ============================================================================ BVH8 reference walker
// Sequential nearest-first walk of the library's compressed BVH8 (node and triangle-record layouts
// of stratum2_b200/csrc/s2_bvh.h, downloaded with s2_get_bvh), counting node and triangle fetches.
// It restates, in plain C++ on the CPU, the traversal order of the library's counted query
// (trav_step: visit a node, test its leaf triangles, descend into the nearest hit child, keep the
// others as one stack group of hit bits): the FP32 slab test of the 8-bit planes with the
// 1.0000004 far-plane padding, the watertight triangle test (isect_tri<float>), closest-hit ties
// to the lowest (instance, primitive).  No alpha test: for scenes without alpha-tested triangles.
// The fetch counts it returns are the algorithmic work of one closest-hit query on this BVH8.
namespace orc {
namespace bvh8 {

struct Group { uint32_t base, bits; };  // child_base, imask | (remaining hit bits << 8)

inline float safe_inv(float d) {
    const float dd = std::fabs(d) < 1e-30f ? std::copysign(1e-30f, d) : d;
    return 1.f / dd;
}
inline float exp2_byte(uint32_t e) { uint32_t b = e << 23; float f; std::memcpy(&f, &b, 4); return f; }
inline float word_f(const uint8_t* p) { float f; std::memcpy(&f, p, 4); return f; }
inline uint32_t word_u(const uint8_t* p) { uint32_t u; std::memcpy(&u, p, 4); return u; }

struct Walk {
    float t, b1, b2;
    uint32_t tri, inst, prim;
    uint32_t nodes, tris;
};

Walk walk(const uint8_t* nodes, const float* tris, const float* ray, bool anyhit) {
    const V3<float> o(ray[0], ray[1], ray[2]), d(ray[4], ray[5], ray[6]);
    const float tmin = ray[3], tmax = ray[7];
    const WRay<float> r = make_wray(o, d, tmin);
    const float inv[3] = {safe_inv(d.x), safe_inv(d.y), safe_inv(d.z)};
    const uint32_t oct = (d.x < 0 ? 1u : 0u) | (d.y < 0 ? 2u : 0u) | (d.z < 0 ? 4u : 0u);
    Walk w{tmax, 0.f, 0.f, 0xffffffffu, 0xffffffffu, 0xffffffffu, 0, 0};
    std::vector<Group> stack;
    uint32_t node = 0;
    while (true) {
        const uint8_t* n = nodes + 128 * (size_t)node;
        w.nodes++;
        const float p[3] = {word_f(n), word_f(n + 4), word_f(n + 8)};
        const uint32_t imask = n[15], child_base = word_u(n + 16), tri_base = word_u(n + 20);
        const uint8_t* meta = n + 24;
        const uint8_t* qlo = n + 32;   // [axis][slot]
        const uint8_t* qhi = n + 56;
        float sc[3], a[3];
        for (int k = 0; k < 3; ++k) { sc[k] = exp2_byte(n[12 + k]) * inv[k]; a[k] = (p[k] - o[k]) * inv[k]; }
        uint32_t hits = 0, trimask = 0;
        for (uint32_t s = 0; s < 8; ++s) {
            float tn[3], tf[3];
            for (int k = 0; k < 3; ++k) {
                const bool neg = inv[k] < 0;
                const float qn = (float)(neg ? qhi[8 * k + s] : qlo[8 * k + s]);
                const float qf = (float)(neg ? qlo[8 * k + s] : qhi[8 * k + s]);
                tn[k] = std::fma(qn, sc[k], a[k]);
                tf[k] = std::fma(qf, sc[k], a[k]);
            }
            const float lo = std::fmax(std::fmax(tn[0], tn[1]), std::fmax(tn[2], tmin));
            const float hi = std::fmin(std::fmin(tf[0], tf[1]), std::fmin(tf[2], w.t)) * 1.0000004f;
            if (lo <= hi) {
                if ((imask >> s) & 1u) hits |= 1u << (s ^ oct);
                else trimask |= ((1u << (meta[s] >> 5)) - 1u) << (meta[s] & 31u);
            }
        }
        for (uint32_t k = 0; k < 32; ++k) {
            if (!((trimask >> k) & 1u)) continue;
            const uint32_t ti = tri_base + k;
            const float* tr = tris + 12 * (size_t)ti;
            const float v[9] = {tr[0], tr[1], tr[2], tr[4], tr[5], tr[6], tr[8], tr[9], tr[10]};
            uint32_t inst, prim;
            std::memcpy(&inst, tr + 3, 4);
            std::memcpy(&prim, tr + 7, 4);
            w.tris++;
            float t, b1, b2;
            if (!isect_tri(r, v, w.t, t, b1, b2)) continue;
            if (anyhit) { w.t = t; w.b1 = b1; w.b2 = b2; w.tri = ti; w.inst = inst; w.prim = prim; return w; }
            if (t < w.t || inst < w.inst || (inst == w.inst && prim < w.prim)) {
                w.t = t; w.b1 = b1; w.b2 = b2; w.tri = ti; w.inst = inst; w.prim = prim;
            }
        }
        auto slot_node = [&](uint32_t base, uint32_t im, uint32_t bit) {
            const uint32_t s = bit ^ oct;
            return base + (uint32_t)__builtin_popcount(im & ((1u << s) - 1u));
        };
        if (hits) {
            const uint32_t b = (uint32_t)__builtin_ctz(hits);
            hits &= hits - 1;
            if (hits) stack.push_back(Group{child_base, imask | (hits << 8)});
            node = slot_node(child_base, imask, b);
            continue;
        }
        if (stack.empty()) return w;
        Group& g = stack.back();
        uint32_t gh = g.bits >> 8;
        const uint32_t b = (uint32_t)__builtin_ctz(gh);
        gh &= gh - 1;
        node = slot_node(g.base, g.bits & 0xffu, b);
        if (gh) g.bits = (g.bits & 0xffu) | (gh << 8);
        else stack.pop_back();
    }
}

}  // namespace bvh8
}  // namespace orc

// rays: n x 8 floats (origin, tmin, direction, tmax); hits: n x 5 words (S2Hit: t, instance,
// primitive, b1, b2); counts: n x 2 (node fetches, triangle fetches).  Returns 0.
extern "C" int oracle_bvh8_trace(const uint8_t* nodes, const float* tris, const float* rays, uint32_t n, int anyhit,
                                 uint32_t* hits, uint32_t* counts) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const orc::bvh8::Walk w = orc::bvh8::walk(nodes, tris, rays + 8 * i, anyhit != 0);
        uint32_t* h = hits + 5 * i;
        std::memcpy(&h[0], &w.t, 4);
        h[1] = w.inst; h[2] = w.prim;
        std::memcpy(&h[3], &w.b1, 4);
        std::memcpy(&h[4], &w.b2, 4);
        counts[2 * i] = w.nodes; counts[2 * i + 1] = w.tris;
    }
    return 0;
}
