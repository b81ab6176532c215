// Device vector math, RNG and packing helpers for the B200 path tracer.
// Each function states the reference shader function it restates (paths relative to the
// Stratum2 source tree).
#pragma once

// fixed-point scale of the batched accumulators: integer sums are independent of the order of the
// (atomic) additions, so batched renders are deterministic
#define S2_FX_SCALE 16777216.0f
#include <cuda_runtime.h>
#include <stdint.h>

#define S2_PI 3.14159265358979323846f
#define S2_INV_PI 0.31830988618379067154f
#define S2_INF __int_as_float(0x7f800000)

#define S2D __device__ __forceinline__

// ---------------------------------------------------------------- float3 arithmetic
S2D float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
S2D float3 f3(float s) { return make_float3(s, s, s); }
S2D float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
S2D float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
S2D float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
S2D float3 operator/(float3 a, float3 b) { return f3(a.x / b.x, a.y / b.y, a.z / b.z); }
S2D float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
S2D float3 operator*(float s, float3 a) { return f3(a.x * s, a.y * s, a.z * s); }
S2D float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
S2D float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
S2D float3& operator+=(float3& a, float3 b) { a = a + b; return a; }
S2D float3& operator*=(float3& a, float3 b) { a = a * b; return a; }
S2D float3& operator*=(float3& a, float s) { a = a * s; return a; }
S2D float3& operator/=(float3& a, float s) { a = a / s; return a; }
S2D float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
S2D float3 cross(float3 a, float3 b) { return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
S2D float length(float3 a) { return sqrtf(dot(a, a)); }
S2D float3 normalize(float3 a) { return a / sqrtf(dot(a, a)); }
S2D float max3(float3 a) { return fmaxf(fmaxf(a.x, a.y), a.z); }
S2D float saturate(float x) { return fminf(fmaxf(x, 0.f), 1.f); }
S2D float lerpf(float a, float b, float t) { return a + (b - a) * t; }
S2D float3 lerp3(float3 a, float3 b, float t) { return a + (b - a) * t; }
S2D float pow2(float x) { return x * x; }
S2D bool any_pos(float3 a) { return a.x > 0 || a.y > 0 || a.z > 0; }
S2D bool all_nonpos(float3 a) { return a.x <= 0 && a.y <= 0 && a.z <= 0; }
S2D bool any_nan(float3 a) { return isnan(a.x) || isnan(a.y) || isnan(a.z); }
S2D float3 sqrt3(float3 a) { return f3(sqrtf(a.x), sqrtf(a.y), sqrtf(a.z)); }
S2D float sgnf(float x) { return x > 0 ? 1.f : (x < 0 ? -1.f : 0.f); }
S2D float3 ld3(const float4 v) { return f3(v.x, v.y, v.z); }

// luminance (src/Shaders/compat/common.h:50)
S2D float luminance(float3 c) { return c.x * 0.2126f + c.y * 0.7152f + c.z * 0.0722f; }

// ---------------------------------------------------------------- RNG (src/Shaders/common/rng.hlsli)
// pcg4d (rng.hlsli:23-35): counter-based 4x32 hash.
S2D uint4 pcg4d(uint4 v) {
    v.x = v.x * 1664525u + 1013904223u; v.y = v.y * 1664525u + 1013904223u;
    v.z = v.z * 1664525u + 1013904223u; v.w = v.w * 1664525u + 1013904223u;
    v.x += v.y * v.w; v.y += v.z * v.x; v.z += v.x * v.y; v.w += v.y * v.z;
    v.x ^= v.x >> 16; v.y ^= v.y >> 16; v.z ^= v.z >> 16; v.w ^= v.w >> 16;
    v.x += v.y * v.w; v.y += v.z * v.x; v.z += v.x * v.y; v.w += v.y * v.z;
    return v;
}
// pcg (rng.hlsli:17-21)
S2D uint32_t pcg_hash(uint32_t v) {
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
// xxhash32 (rng.hlsli:5-13)
S2D uint32_t xxhash32(uint32_t p) {
    const uint32_t P2 = 2246822519U, P3 = 3266489917U, P4 = 668265263U, P5 = 374761393U;
    uint32_t h = p + P5;
    h = P4 * ((h << 17) | (h >> 15));
    h = P2 * (h ^ (h >> 15));
    h = P3 * (h ^ (h >> 13));
    return h ^ (h >> 16);
}
// u32 -> [0,1) float from the top 23 bits (rng.hlsli:58-60)
S2D float u2f(uint32_t u) { return __uint_as_float(0x3f800000u | (u >> 9)) - 1.f; }

// RandomSampler (rng.hlsli:39-56): state (pixel.x, pixel.y, seed, counter); next() increments
// the counter and hashes.  The PCG32 variant (flag S2_FLAG_PCG32) keeps a 64-bit LCG state
// seeded from (pixel, sample) and draws four 32-bit outputs per next().
struct Rng {
    uint32_t px, py, seed, ctr;  // pcg4d state; for PCG32: (state_lo, state_hi, inc_lo, -)
    bool pcg32;
    S2D uint4 next() {
        if (!pcg32) {
            ctr++;
            return pcg4d(make_uint4(px, py, seed, ctr));
        }
        uint4 r;
        r.x = pcg32_step(); r.y = pcg32_step(); r.z = pcg32_step(); r.w = pcg32_step();
        return r;
    }
    // advance by one next() without hashing (pcg4d is counter based)
    S2D void skip() {
        if (!pcg32) { ctr++; return; }
        pcg32_step(); pcg32_step(); pcg32_step(); pcg32_step();
    }
    S2D float4 next_float() {
        uint4 u = next();
        return make_float4(u2f(u.x), u2f(u.y), u2f(u.z), u2f(u.w));
    }
    // PCG32 (O'Neill 2014, XSH-RR output of a 64-bit LCG)
    S2D uint32_t pcg32_step() {
        unsigned long long state = ((unsigned long long)py << 32) | px;
        unsigned long long inc = ((unsigned long long)ctr << 32) | seed;
        unsigned long long old = state;
        state = old * 6364136223846793005ULL + (inc | 1ULL);
        px = (uint32_t)state; py = (uint32_t)(state >> 32);
        uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
    }
};
S2D Rng make_rng(uint32_t pixel_x, uint32_t pixel_y, uint32_t seed, bool pcg32) {
    Rng r;
    r.pcg32 = pcg32;
    if (!pcg32) { r.px = pixel_x; r.py = pixel_y; r.seed = seed; r.ctr = 0; return r; }
    // stream = (pixel), initial state from (sample): standard pcg32_srandom
    const unsigned long long initstate = ((unsigned long long)seed << 32) ^ 0x853c49e6748fea9bULL;
    const unsigned long long initseq = ((unsigned long long)pixel_y << 32) | pixel_x;
    const unsigned long long inc = (initseq << 1u) | 1u;
    r.seed = (uint32_t)inc; r.ctr = (uint32_t)(inc >> 32);
    r.px = 0; r.py = 0;
    r.pcg32_step();
    unsigned long long st = (((unsigned long long)r.py << 32) | r.px) + initstate;
    r.px = (uint32_t)st; r.py = (uint32_t)(st >> 32);
    r.pcg32_step();
    return r;
}

// ---------------------------------------------------------------- normal packing
// Octahedral map (src/Shaders/common/common.hlsli:5-22) stored as R16G16_SNORM
// (D3DX_DXGIFormatConvert.inl: D3DX_FLOAT2_to_R16G16_SNORM / D3DX_R16G16_SNORM_to_FLOAT2).
// D3DX_FLOAT_to_INT: a separate multiply and add (explicitly rounded, so no contraction into an
// FMA changes the result with the surrounding code)
S2D int snorm_from_float(float v) {
    if (isnan(v)) v = 0.f;
    v = fminf(fmaxf(v, -1.f), 1.f);
    return (int)truncf(__fadd_rn(__fmul_rn(v, 32767.f), v >= 0 ? 0.5f : -0.5f));
}
// The packing divides and normalises with IEEE-rounded intrinsics: ray directions go through this
// quantisation, so it stays exact whatever the compiler's division and square-root settings.
S2D float float_from_snorm(int v) { return fmaxf(__fdiv_rn((float)v, 32767.f), -1.f); }
S2D float3 normalize_ieee(float3 a) {
    const float l = __fsqrt_rn(dot(a, a));
    return f3(__fdiv_rn(a.x, l), __fdiv_rn(a.y, l), __fdiv_rn(a.z, l));
}
S2D uint32_t pack_normal(float3 v) {
    const float inv = __fdiv_rn(1.f, fabsf(v.x) + fabsf(v.y) + fabsf(v.z));
    float px = v.x * inv, py = v.y * inv;
    if (v.z <= 0) {
        const float ox = (1.f - fabsf(py)) * (px >= 0 ? 1.f : -1.f);
        const float oy = (1.f - fabsf(px)) * (py >= 0 ? 1.f : -1.f);
        px = ox; py = oy;
    }
    return ((uint32_t)snorm_from_float(px) & 0xffffu) | ((uint32_t)snorm_from_float(py) << 16);
}
S2D float3 unpack_normal(uint32_t p) {
    const float x = float_from_snorm((int)(p << 16) >> 16);
    const float y = float_from_snorm((int)(p & 0xffff0000u) >> 16);
    float3 v = f3(x, y, 1.f - (fabsf(x) + fabsf(y)));
    if (v.z < 0) {
        const float ox = (1.f - fabsf(v.y)) * (v.x >= 0 ? 1.f : -1.f);
        const float oy = (1.f - fabsf(v.x)) * (v.y >= 0 ? 1.f : -1.f);
        v.x = ox; v.y = oy;
    }
    return normalize_ieee(v);
}

// makeOrthonormal (common.hlsli:24-34): rows t, b, n
S2D void make_orthonormal(float3 N, float3& t, float3& b) {
    if (N.x != N.y || N.x != N.z) t = f3(N.z - N.y, N.x - N.z, N.y - N.x);
    else t = f3(N.z - N.y, N.x + N.z, -N.y - N.x);
    t = normalize(t);
    b = cross(N, t);
}

// sampling helpers (common.hlsli:36-76)
S2D float2 sample_uniform_triangle(float u1, float u2) {
    const float a = sqrtf(u1);
    return make_float2(1.f - a, a * u2);
}
S2D float3 sample_uniform_sphere(float u1, float u2) {
    const float z = u2 * 2.f - 1.f;
    const float r = sqrtf(fmaxf(1.f - z * z, 0.f));
    const float phi = 2.f * S2_PI * u1;
    return f3(r * cosf(phi), r * sinf(phi), z);
}
S2D float2 sample_concentric_disc(float u1, float u2) {
    const float ox = 2.f * u1 - 1.f, oy = 2.f * u2 - 1.f;
    if (ox == 0 && oy == 0) return make_float2(0.f, 0.f);
    float theta, r;
    if (fabsf(ox) > fabsf(oy)) { r = ox; theta = (S2_PI / 4.f) * (oy / ox); }
    else { r = oy; theta = S2_PI / 2.f - (S2_PI / 4.f) * (ox / oy); }
    return make_float2(r * cosf(theta), r * sinf(theta));
}
S2D float3 sample_cos_hemisphere(float u1, float u2) {
    const float2 xy = sample_concentric_disc(u1, u2);
    return f3(xy.x, xy.y, sqrtf(fmaxf(0.f, 1.f - (xy.x * xy.x + xy.y * xy.y))));
}
S2D float cos_hemisphere_pdfw(float c) { return fmaxf(c, 0.f) / S2_PI; }

// rayOffset (src/Shaders/common/intersection.hlsli:17-32), Waechter & Binder 2019
S2D float offset_axis(float p, float n) {
    const float origin = 1.f / 32.f, float_scale = 1.f / 65536.f, int_scale = 256.f;
    const int of_i = (int)(int_scale * n);
    return fabsf(p) < origin ? p + float_scale * n : __int_as_float(__float_as_int(p) + (p < 0 ? -of_i : of_i));
}
S2D float3 ray_offset(float3 P, float3 Ng) { return f3(offset_axis(P.x, Ng.x), offset_axis(P.y, Ng.y), offset_axis(P.z, Ng.z)); }
S2D float3 ray_offset(float3 P, float3 Ng, float3 dir) { return ray_offset(P, dot(Ng, dir) < 0 ? -Ng : Ng); }
// AdjustIntersectionDistance (intersection.hlsli:65)
S2D float adjust_distance(float d) { return fmaxf(d * 0.99f, d - 1e-2f); }

// spherical uv (src/Shaders/compat/common.h:129-142)
S2D float stable_atan2(float y, float x) {
    return x == 0.f ? (y == 0.f ? 0.f : (y < 0 ? -S2_PI / 2 : S2_PI / 2)) : atan2f(y, x);
}
S2D float2 cartesian_to_spherical_uv(float3 v) {
    const float theta = stable_atan2(v.z, v.x);
    return make_float2(theta * S2_INV_PI * 0.5f + 0.5f, acosf(fminf(fmaxf(v.y, -1.f), 1.f)) * S2_INV_PI);
}
S2D float3 spherical_uv_to_cartesian(float2 uv) {
    const float u = (uv.x * 2.f - 1.f) * S2_PI, v = uv.y * S2_PI;
    const float s = sinf(v);
    return f3(s * cosf(u), cosf(v), s * sinf(u));
}

// power heuristic (src/Shaders/kernels/testrenderer.slang:284-290)
S2D float mis2(float a) { return a * a; }
S2D float mis(float a, float b) { const float a2 = a * a; return a2 / (a2 + b * b); }
