// ORACLE -- test infrastructure only.  The reference's own shader math (Stratum2's
// src/Shaders/common/rng.hlsli, common.hlsli with D3DX_DXGIFormatConvert.inl, and microfacet.hlsli)
// compiled as host C++ over hlsl_shim.h, exposed so tests can pin the oracle and the device code to
// it.  oracle/build_oracle.py writes the host-compilable copies of those files into oracle/_ref/gen/
// (the edits are listed there) and builds this file into oracle/_ref/libref_shader.so; nothing here
// is shipped in the product.
#include <cstdint>

#include "hlsl_shim.h"

using namespace hlsl;
#define precise

#include "_ref/gen/rng.hlsli"
#include "_ref/gen/common.hlsli"
#include "_ref/gen/microfacet.hlsli"

#undef precise

// Function ids and per-entry layouts of ref_shader_math (inputs: REF_IN doubles per entry, outputs:
// REF_OUT doubles per entry; unsigned integers travel as exact doubles).
enum {
    REF_XXHASH32 = 0,       // in u                         out h                    (rng.hlsli:5-13)
    REF_PCG = 1,            // in u                         out h                    (rng.hlsli:17-21)
    REF_PCG4D = 2,          // in u4                        out u4                   (rng.hlsli:23-35)
    REF_NEXT_FLOAT = 3,     // in px py seed offset         out 4 floats of the first nextFloat() (rng.hlsli:39-60)
    REF_PACK_NORMAL = 4,    // in xyz                       out packed               (common.hlsli:18-20)
    REF_UNPACK_NORMAL = 5,  // in packed                    out xyz                  (common.hlsli:21-23)
    REF_GTR1 = 6,           // in n.h alpha                 out D                    (microfacet.hlsli:64-69)
    REF_GTR2_ANISO = 7,     // in h.xyz ax ay               out D                    (microfacet.hlsli:79-83)
    REF_SMITH_GTR2 = 8,     // in v.xyz ax ay               out G1                   (microfacet.hlsli:104-110)
    REF_SMITH_GTR1 = 9,     // in v.xyz                     out G1                   (microfacet.hlsli:112-114)
    REF_VNDF = 10,          // in in.xyz ax ay u1 u2        out h.xyz                (microfacet.hlsli:148-179)
    REF_SCHLICK = 11,       // in F0 cos                    out F                    (microfacet.hlsli:25-27)
    REF_FRESNEL_DIEL = 12,  // in n.i eta                   out F                    (microfacet.hlsli:55-62)
    REF_CONCENTRIC = 13,    // in u1 u2                     out xy                   (common.hlsli:47-67)
    REF_COS_HEMI = 14,      // in u1 u2                     out xyz                  (common.hlsli:72-75)
    REF_UNIFORM_SPHERE = 15,// in u1 u2                     out xyz                  (common.hlsli:40-45)
    REF_UNIFORM_TRI = 16,   // in u1 u2                     out b1 b2                (common.hlsli:36-39)
    REF_ORTHONORMAL = 17,   // in n.xyz                     out rows r0 r1 r2        (common.hlsli:24-34)
    REF_COUNT = 18
};
constexpr int REF_IN = 8, REF_OUT = 9;

extern "C" {

int ref_shader_math(int fn, const double* in, uint32_t n, double* out) {
    if (fn < 0 || fn >= REF_COUNT) return -1;
    for (uint32_t k = 0; k < n; ++k) {
        const double* a = in + (size_t)REF_IN * k;
        double* o = out + (size_t)REF_OUT * k;
        auto f = [&](int i) { return (float)a[i]; };
        auto u = [&](int i) { return (uint)a[i]; };
        auto put3 = [&](const float3& v, int at = 0) { o[at] = v.x; o[at + 1] = v.y; o[at + 2] = v.z; };
        switch (fn) {
            case REF_XXHASH32: o[0] = xxhash32(u(0)); break;
            case REF_PCG: o[0] = pcg(u(0)); break;
            case REF_PCG4D: {
                const uint4 r = pcg4d(uint4(u(0), u(1), u(2), u(3)));
                o[0] = r.x; o[1] = r.y; o[2] = r.z; o[3] = r.w;
                break;
            }
            case REF_NEXT_FLOAT: {
                RandomSampler rs(u(2), uint2(u(0), u(1)), u(3));
                const float4 r = rs.nextFloat();
                o[0] = r.x; o[1] = r.y; o[2] = r.z; o[3] = r.w;
                break;
            }
            case REF_PACK_NORMAL: o[0] = packNormal(float3(f(0), f(1), f(2))); break;
            case REF_UNPACK_NORMAL: put3(unpackNormal(u(0))); break;
            case REF_GTR1: o[0] = GTR1(f(0), f(1)); break;
            case REF_GTR2_ANISO: o[0] = GTR2(float3(f(0), f(1), f(2)), f(3), f(4)); break;
            case REF_SMITH_GTR2: o[0] = smith_masking_gtr2(float3(f(0), f(1), f(2)), f(3), f(4)); break;
            case REF_SMITH_GTR1: o[0] = smith_masking_gtr1(float3(f(0), f(1), f(2))); break;
            case REF_VNDF: put3(sample_visible_normals(float3(f(0), f(1), f(2)), f(3), f(4), float2(f(5), f(6)))); break;
            case REF_SCHLICK: o[0] = schlick_fresnel(f(0), f(1)); break;
            case REF_FRESNEL_DIEL: o[0] = fresnel_dielectric(f(0), f(1)); break;
            case REF_CONCENTRIC: { const float2 r = sampleConcentricDisc(f(0), f(1)); o[0] = r.x; o[1] = r.y; break; }
            case REF_COS_HEMI: put3(sampleCosHemisphere(f(0), f(1))); break;
            case REF_UNIFORM_SPHERE: put3(sampleUniformSphere(f(0), f(1))); break;
            case REF_UNIFORM_TRI: { const float2 r = sampleUniformTriangle(f(0), f(1)); o[0] = r.x; o[1] = r.y; break; }
            case REF_ORTHONORMAL: {
                const float3x3 m = makeOrthonormal(float3(f(0), f(1), f(2)));
                put3(m[0], 0); put3(m[1], 3); put3(m[2], 6);
                break;
            }
        }
    }
    return 0;
}

}  // extern "C"
