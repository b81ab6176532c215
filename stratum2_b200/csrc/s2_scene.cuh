// Device-resident scene: the reference's SceneParameters (src/Shaders/common/scene.hlsli:6-41)
// as flat device pointers, plus the BVH8 that replaces its acceleration structure.
#pragma once
#include "s2_math.cuh"

#define S2_MAX_IMAGE_LEVELS 16

struct DevImage {
    const float4* texels;       // level 0, RGBA (missing channels read as 0, alpha 1)
    uint32_t width, height;
    // luminance pyramid for hierarchical sampling (levels 0..levels-1), only for environment maps
    const float* lum;           // concatenated levels
    uint32_t levels;
    uint32_t lum_offset[S2_MAX_IMAGE_LEVELS];
    uint32_t lw[S2_MAX_IMAGE_LEVELS], lh[S2_MAX_IMAGE_LEVELS];
    // Precomputed hierarchical-sampling tables (only when every level is an exact halving, so a
    // texel of the finest sampled level determines its 2x2 block at every coarser level):
    //   quad: per level, per 2x2 block (block x = cx/2, y = cy/2) the normalised probabilities of
    //         its four texels, or x = -1 where their luminance-weighted sum is below 1e-6;
    //   pdf:  per texel of the finest sampled level, the texel pdf of SampleTexelPdf.
    const float4* quad;
    uint32_t quad_offset[S2_MAX_IMAGE_LEVELS];
    uint32_t qw[S2_MAX_IMAGE_LEVELS];
    const float* pdf;
    uint32_t pdf_level;
    uint32_t nested;
};

struct DevScene {
    // BVH8
    const uint4* nodes;
    const float4* tris;
    uint32_t tri_count;
    // instances (compat/scene.h:30-58), transforms (compat/transform.h:7)
    const uint2* instances;
    const uint32_t* prim_counts;       // 32-bit primitive counts
    const float4* transforms;          // 3 rows per instance
    const float4* inv_transforms;
    const float4* motion_transforms;
    uint32_t instance_count;
    // vertex data (compat/scene.h:89-132; scene.hlsli:43-70)
    const uint32_t* vertex_infos;      // 8 words per MeshVertexInfo
    const uint8_t* const* vbufs;
    uint32_t vbuf_count;
    // materials (material_data.h, Material.hpp:22-38)
    const uint8_t* material_data;
    uint32_t material_bytes;
    // lights (Scene.cpp:441-491)
    const uint32_t* light_instance_map;
    const uint32_t* instance_light_map;
    uint32_t light_count;
    // power-proportional light pick (S2_FLAG_LIGHT_POWER_PICK; no counterpart in the reference, whose
    // pick is uniform): Walker alias table over the lights {threshold, alias index as float bits}
    // and each light's pick probability; light_power_pick is set per render call
    const float2* light_alias;
    const float* light_pick_pdf;
    uint32_t light_power_pick;
    // baked light triangles for that mode: per light {first record, triangle count}; per triangle
    // four float4 {v0, area}, {v1 - v0, emission r}, {v2 - v0, emission g}, {geometric normal,
    // emission b}, world space; area <= 0 marks a triangle sampled through make_shading instead
    // (vertex normals, which may flip the geometric normal, or an emission texture)
    const uint2* light_tri_range;
    const float4* light_tris;
    uint32_t env_address;              // 0xffffffff = none
    float env_sample_prob;
    // images
    const DevImage* images;
    uint32_t image_count;
    // S2_FLAG_ENV_FOOTPRINT_PDF: the environment image's descriptor with sampling tables built from
    // the per-texel maximum of its bilinear luminance (same texels); env_fp_on is set per render call
    const DevImage* env_fp;
    uint32_t env_fp_on;
    float4 scene_sphere;
    // ray-coherence keys: the BVH root box as origin and 8 / extent per axis (zero: no BVH)
    float4 key_lo, key_scale;
    // baked shading records, four float4 per BVH triangle (k_bake_shading; null: none, or switched
    // off by S2Tuning.shade_records)
    const float4* shade_recs;
};

// Ray-coherence key: Morton code of the origin's cell in an 8^3 grid over the BVH root box
// (9 bits) above the direction octant (3 bits), 12 bits in all.
S2D uint32_t ray_key(const DevScene& s, float3 o, float3 d) {
    const int cx = min(max((int)((o.x - s.key_lo.x) * s.key_scale.x), 0), 7);
    const int cy = min(max((int)((o.y - s.key_lo.y) * s.key_scale.y), 0), 7);
    const int cz = min(max((int)((o.z - s.key_lo.z) * s.key_scale.z), 0), 7);
    uint32_t m = 0;
#pragma unroll
    for (int b = 0; b < 3; ++b) m |= (((cx >> b) & 1) << (3 * b + 2)) | (((cy >> b) & 1) << (3 * b + 1)) | (((cz >> b) & 1) << (3 * b));
    return (m << 3) | (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
}

// ---- transforms (TransformData: row-major 3x4)
S2D float3 xform_point(const float4* m, float3 p) {
    const float4 r0 = m[0], r1 = m[1], r2 = m[2];
    return f3(r0.x * p.x + r0.y * p.y + r0.z * p.z + r0.w,
              r1.x * p.x + r1.y * p.y + r1.z * p.z + r1.w,
              r2.x * p.x + r2.y * p.y + r2.z * p.z + r2.w);
}
S2D float3 xform_vector(const float4* m, float3 v) {
    const float4 r0 = m[0], r1 = m[1], r2 = m[2];
    return f3(r0.x * v.x + r0.y * v.y + r0.z * v.z,
              r1.x * v.x + r1.y * v.y + r1.z * v.z,
              r2.x * v.x + r2.y * v.y + r2.z * v.z);
}

// ---- byte-address loads
S2D uint32_t ld_u32(const uint8_t* base, uint32_t off) { return *(const uint32_t*)(base + off); }
S2D float ld_f32(const uint8_t* base, uint32_t off) { return *(const float*)(base + off); }

// MeshVertexInfo accessors (compat/scene.h:95-108)
struct VInfo { uint32_t w[8]; };
S2D VInfo load_vinfo(const DevScene& s, uint32_t idx) {
    const uint4* p = (const uint4*)(s.vertex_infos + 8 * (size_t)idx);
    const uint4 a = p[0], b = p[1];
    VInfo v; v.w[0] = a.x; v.w[1] = a.y; v.w[2] = a.z; v.w[3] = a.w; v.w[4] = b.x; v.w[5] = b.y; v.w[6] = b.z; v.w[7] = b.w;
    return v;
}
S2D uint32_t vi_index_buffer(const VInfo& v) { return v.w[0] & 0xffffu; }
S2D uint32_t vi_position_buffer(const VInfo& v) { return v.w[0] >> 16; }
S2D uint32_t vi_normal_buffer(const VInfo& v) { return v.w[1] & 0xffffu; }
S2D uint32_t vi_texcoord_buffer(const VInfo& v) { return v.w[1] >> 16; }
S2D uint32_t vi_index_stride(const VInfo& v) { return v.w[2] & 0xffu; }
S2D uint32_t vi_position_stride(const VInfo& v) { return (v.w[2] >> 8) & 0xffu; }
S2D uint32_t vi_normal_stride(const VInfo& v) { return (v.w[2] >> 16) & 0xffu; }
S2D uint32_t vi_texcoord_stride(const VInfo& v) { return v.w[2] >> 24; }
S2D uint32_t vi_index_offset(const VInfo& v) { return v.w[4]; }
S2D uint32_t vi_position_offset(const VInfo& v) { return v.w[5]; }
S2D uint32_t vi_normal_offset(const VInfo& v) { return v.w[6]; }
S2D uint32_t vi_texcoord_offset(const VInfo& v) { return v.w[7]; }

// LoadTriangleIndices (scene.hlsli:43-62)
S2D uint3 load_triangle_indices(const uint8_t* ib, uint32_t offset, uint32_t stride, uint32_t prim) {
    const uint32_t off = offset + prim * 3u * stride;
    if (stride == 2) {
        const uint32_t al = off & ~3u;
        const uint32_t w0 = ld_u32(ib, al), w1 = ld_u32(ib, al + 4);
        if (al == off) return make_uint3(w0 & 0xffffu, w0 >> 16, w1 & 0xffffu);
        return make_uint3(w0 >> 16, w1 & 0xffffu, w1 >> 16);
    }
    return make_uint3(ld_u32(ib, off), ld_u32(ib, off + 4), ld_u32(ib, off + 8));
}
S2D float3 load_f3(const uint8_t* b, uint32_t offset, uint32_t stride, uint32_t i) {
    const uint32_t o = offset + stride * i;
    return f3(ld_f32(b, o), ld_f32(b, o + 4), ld_f32(b, o + 8));
}
S2D float2 load_f2(const uint8_t* b, uint32_t offset, uint32_t stride, uint32_t i) {
    const uint32_t o = offset + stride * i;
    return make_float2(ld_f32(b, o), ld_f32(b, o + 4));
}

// ---- images: bilinear, repeat addressing, level 0 (SampleLevel(..., 0) with a linear/repeat
// sampler, TestRenderer.cpp:54-57)
S2D float4 sample_image(const DevImage& im, float2 uv) {
    const float x = uv.x * im.width - 0.5f, y = uv.y * im.height - 0.5f;
    const float fx = floorf(x), fy = floorf(y);
    const float ax = x - fx, ay = y - fy;
    int x0 = (int)fx, y0 = (int)fy;
    const int W = (int)im.width, H = (int)im.height;
    x0 %= W; if (x0 < 0) x0 += W;
    y0 %= H; if (y0 < 0) y0 += H;
    const int x1 = (x0 + 1) % W, y1 = (y0 + 1) % H;
    const float4 a = im.texels[(size_t)y0 * W + x0], b = im.texels[(size_t)y0 * W + x1];
    const float4 c = im.texels[(size_t)y1 * W + x0], d = im.texels[(size_t)y1 * W + x1];
    const float w00 = (1 - ax) * (1 - ay), w10 = ax * (1 - ay), w01 = (1 - ax) * ay, w11 = ax * ay;
    return make_float4(a.x * w00 + b.x * w10 + c.x * w01 + d.x * w11,
                       a.y * w00 + b.y * w10 + c.y * w01 + d.y * w11,
                       a.z * w00 + b.z * w10 + c.z * w01 + d.z * w11,
                       a.w * w00 + b.w * w10 + c.w * w01 + d.w * w11);
}

// The candidate test of a non-opaque triangle (intersection.hlsli:125-146, gAlphaTest): the
// material's alpha-mask image (getMaterialAlphaMask, material.hlsli:72-76: index and cutoff at
// bytes 48 and 52 of the record) sampled at the hit's texture coordinate, level 0, red channel,
// accepted when >= cutoff.  `on` false (S2_FLAG_ALPHA_TEST_OFF) accepts every triangle.
struct SceneAlphaTest {
    const DevScene* s;
    bool on;
    S2D bool operator()(uint32_t inst, uint32_t prim, float b1, float b2) const {
        if (!on) return true;
        const DevScene& sc = *s;
        const uint32_t mat = sc.instances[inst].x >> 4;
        const uint2 am = *(const uint2*)(sc.material_data + mat + 48);
        if (am.x >= sc.image_count) return true;
        const VInfo vi = load_vinfo(sc, sc.instances[inst].y & 0xffffu);
        float2 uv = make_float2(0.f, 0.f);
        const uint32_t tb = vi_texcoord_buffer(vi);
        if (tb < sc.vbuf_count) {
            const uint3 tri = load_triangle_indices(sc.vbufs[vi_index_buffer(vi)], vi_index_offset(vi), vi_index_stride(vi), prim);
            const uint8_t* tbuf = sc.vbufs[tb];
            const uint32_t to = vi_texcoord_offset(vi), ts = vi_texcoord_stride(vi);
            const float2 t0 = load_f2(tbuf, to, ts, tri.x), t1 = load_f2(tbuf, to, ts, tri.y), t2 = load_f2(tbuf, to, ts, tri.z);
            uv = make_float2(t0.x + (t1.x - t0.x) * b1 + (t2.x - t0.x) * b2, t0.y + (t1.y - t0.y) * b1 + (t2.y - t0.y) * b2);
        }
        return sample_image(sc.images[am.x], uv).x >= __uint_as_float(am.y);
    }
};
