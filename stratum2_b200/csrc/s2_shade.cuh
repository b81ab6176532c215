// Device shading: hit reconstruction, materials, BSDFs and light sampling for the wavefront
// path tracer.  Each function restates the reference shader function it cites (paths relative
// to the Stratum2 source tree).
#pragma once
#include <cuda_fp16.h>

#include "s2_scene.cuh"

// f32tof16 / f16tof32 round trip: the reference keeps mDirPdfW, mIntersectionDistance and
// mIntersectionPdfA of its PathState as half floats (testrenderer.slang:75-97).
S2D float half_round(float x) { return __half2float(__float2half_rn(x)); }

// power heuristic with the limit value for an overflowed (infinite) half-precision pdf
S2D float mis_w(float a, float b) {
    if (isinf(a)) return isinf(b) ? 0.5f : 1.f;
    const float a2 = a * a;
    return a2 / (a2 + b * b);
}

// ---------------------------------------------------------------- materials
// PackedMaterialData (src/Shaders/compat/material_data.h:12-73)
S2D float un8(uint32_t w, int shift) { return (float)((w >> shift) & 0xffu) / 255.f; }
S2D uint32_t pk8(float v) { v = saturate(v); return (uint32_t)floorf(v * 255.f + 0.5f); }

struct Mat {
    uint32_t w[4];
    float escale;
    S2D float3 base() const { return f3(un8(w[0], 0), un8(w[0], 8), un8(w[0], 16)); }
    S2D float3 emission() const { return f3(un8(w[1], 0), un8(w[1], 8), un8(w[1], 16)) * escale; }
    S2D float specular() const { return un8(w[0], 24); }
    S2D float sheen() const { return un8(w[1], 24); }
    S2D float metallic() const { return un8(w[2], 0); }
    S2D float roughness() const { return un8(w[2], 8); }
    S2D float anisotropic() const { return un8(w[2], 16); }
    S2D float subsurface() const { return un8(w[2], 24); }
    S2D float clearcoat() const { return un8(w[3], 0); }
    S2D float clearcoat_gloss() const { return un8(w[3], 8); }
    S2D float transmission() const { return un8(w[3], 16); }
    S2D float eta1() const { return un8(w[3], 24) + 1.f; }
    S2D void set_base(float3 c) { w[0] = (w[0] & 0xff000000u) | pk8(c.x) | pk8(c.y) << 8 | pk8(c.z) << 16; }
    S2D void set_emission(float3 c) {
        escale = max3(c);
        c = c / escale;
        const uint32_t r = isnan(c.x) ? 0u : pk8(c.x), g = isnan(c.y) ? 0u : pk8(c.y), b = isnan(c.z) ? 0u : pk8(c.z);
        w[1] = (w[1] & 0xff000000u) | r | g << 8 | b << 16;
    }
};

// LoadMaterial (src/Shaders/common/material.hlsli:15-46), texture lookups at level 0
S2D Mat load_material(const DevScene& s, uint32_t addr, float2 uv) {
    Mat m;
    const uint4 a = *(const uint4*)(s.material_data + addr);
    const uint4 img = *(const uint4*)(s.material_data + addr + 16);
    m.w[0] = a.x; m.w[1] = a.y; m.w[2] = a.z; m.w[3] = a.w;
    m.escale = ld_f32(s.material_data, addr + 32);
    const uint32_t n = s.image_count;
    if (img.x < n) { const float4 t = sample_image(s.images[img.x], uv); m.set_base(m.base() * f3(t.x, t.y, t.z)); }
    if (img.y < n) { const float4 t = sample_image(s.images[img.y], uv); m.set_emission(m.emission() * f3(t.x, t.y, t.z)); }
    if (img.z < n) {
        const float4 t = sample_image(s.images[img.z], uv);
        const float x = un8(m.w[2], 0) * t.x, y = 1.f - (1.f - un8(m.w[2], 8)) * (1.f - t.y);
        const float z = un8(m.w[2], 16) * t.z, q = un8(m.w[2], 24) * t.w;
        m.w[2] = pk8(x) | pk8(y) << 8 | pk8(z) << 16 | pk8(q) << 24;
    }
    if (img.w < n) {
        const float4 t = sample_image(s.images[img.w], uv);
        m.w[3] = pk8(un8(m.w[3], 0) * t.x) | pk8(un8(m.w[3], 8) * t.y) << 8 | pk8(un8(m.w[3], 16) * t.z) << 16 | pk8(un8(m.w[3], 24) * t.w) << 24;
    }
    return m;
}

// ---------------------------------------------------------------- shading data
// ShadingData (compat/scene.h:186-198) with the packed normals already unpacked.
struct SD {
    float3 pos;
    uint32_t mat;
    uint32_t ng, ns, tg;     // packed geometry normal, shading normal, tangent
    float area;
    float2 uv;
    float3 n, t, b, gn;      // unpacked shading frame and geometry normal
    S2D float3 to_local(float3 v) const { return f3(dot(v, t), dot(v, b), dot(v, n)); }
    S2D float3 to_world(float3 v) const { return t * v.x + b * v.y + n * v.z; }
    // shadingNormalCorrection<false> (shading_data.hlsli:35-55)
    S2D float snc(float3 in, float3 out) const {
        const float3 lg = to_local(gn);
        const float a = dot(lg, in), c = dot(lg, out);
        if (sgnf(c) != sgnf(out.z) || sgnf(a) != sgnf(in.z)) return 0.f;
        return 1.f;
    }
};

// Explicitly rounded vector helpers for the per-triangle shading terms: no multiply-add of these
// is contracted into an FMA, so the terms are the same wherever make_shading is inlined (the
// baked shading records hold them and must equal the gathered path bit for bit).
S2D float3 xform_vector_rn(const float4* m, float3 v) {
    const float4 r0 = m[0], r1 = m[1], r2 = m[2];
    return f3(__fadd_rn(__fadd_rn(__fmul_rn(r0.x, v.x), __fmul_rn(r0.y, v.y)), __fmul_rn(r0.z, v.z)),
              __fadd_rn(__fadd_rn(__fmul_rn(r1.x, v.x), __fmul_rn(r1.y, v.y)), __fmul_rn(r1.z, v.z)),
              __fadd_rn(__fadd_rn(__fmul_rn(r2.x, v.x), __fmul_rn(r2.y, v.y)), __fmul_rn(r2.z, v.z)));
}
S2D float3 cross_rn(float3 a, float3 b) {
    return f3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
              __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
S2D float length_rn(float3 a) {
    return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(a.x, a.x), __fmul_rn(a.y, a.y)), __fmul_rn(a.z, a.z)));
}
S2D float3 div_rn(float3 a, float s) { return f3(__fdiv_rn(a.x, s), __fdiv_rn(a.y, s), __fdiv_rn(a.z, s)); }
S2D float3 normalize_rn(float3 a) { return div_rn(a, length_rn(a)); }
// makeOrthonormal's first row (common.hlsli:24-34), explicitly rounded
S2D float3 orthonormal_t_rn(float3 N) {
    const float3 t = (N.x != N.y || N.x != N.z) ? f3(__fsub_rn(N.z, N.y), __fsub_rn(N.x, N.z), __fsub_rn(N.y, N.x))
                                                 : f3(__fsub_rn(N.z, N.y), __fadd_rn(N.x, N.z), __fsub_rn(-N.y, N.x));
    return normalize_rn(t);
}

// makeTriangleShadingData (shading_data.hlsli:59-151): gathers indices and attributes through
// MeshVertexInfo (scene.hlsli:43-70) and applies the instance transform.  shading_terms fills
// everything but the hit position and the unpacked frame, and returns the object-space vertex v0
// and edges v1 - v0, v2 - v0; shading_finish adds those from the barycentrics.
S2D void shading_terms(const DevScene& s, uint32_t inst, uint32_t prim, float b1, float b2, bool shading_normals, SD& r,
                       float3& v0, float3& e1, float3& e2) {
    const uint2 id = s.instances[inst];
    r.mat = id.x >> 4;
    const float4* M = s.transforms + 3 * (size_t)inst;
    const VInfo vi = load_vinfo(s, id.y & 0xffffu);
    const uint3 tri = load_triangle_indices(s.vbufs[vi_index_buffer(vi)], vi_index_offset(vi), vi_index_stride(vi), prim);
    const uint8_t* pb = s.vbufs[vi_position_buffer(vi)];
    const uint32_t po = vi_position_offset(vi), ps = vi_position_stride(vi);
    v0 = load_f3(pb, po, ps, tri.x);
    const float3 v1 = load_f3(pb, po, ps, tri.y), v2 = load_f3(pb, po, ps, tri.z);
    e1 = v1 - v0;
    e2 = v2 - v0;
    const float3 dPds = xform_vector_rn(M, v0 - v2), dPdt = xform_vector_rn(M, v1 - v2);
    float3 gn = cross_rn(dPds, dPdt);
    const float area2 = length_rn(gn);
    gn = div_rn(gn, area2);
    r.ng = pack_normal(gn);
    r.area = __fmul_rn(area2, 0.5f);
    float2 t0 = make_float2(0.f, 0.f), t1 = t0, t2 = t0;
    const uint32_t tb = vi_texcoord_buffer(vi);
    if (tb < s.vbuf_count) {
        const uint8_t* tbuf = s.vbufs[tb];
        const uint32_t to = vi_texcoord_offset(vi), ts = vi_texcoord_stride(vi);
        t0 = load_f2(tbuf, to, ts, tri.x); t1 = load_f2(tbuf, to, ts, tri.y); t2 = load_f2(tbuf, to, ts, tri.z);
    }
    const float2 duvds = make_float2(t2.x - t0.x, t2.y - t0.y), duvdt = make_float2(t2.x - t1.x, t2.y - t1.y);
    r.uv = make_float2(t0.x + (t1.x - t0.x) * b1 + duvds.x * b2, t0.y + (t1.y - t0.y) * b1 + duvds.y * b2);
    const float det = duvds.x * duvdt.y - duvdt.x * duvds.y;
    float3 dPdu;
    if (det != 0.f) {
        const float idet = 1.f / det;
        const float dsdu = duvdt.y * idet, dtdu = -duvds.y * idet;
        dPdu = -(dPds * dsdu + dPdt * dtdu);
    } else {
        dPdu = orthonormal_t_rn(gn);
    }
    bool valid = false;
    float3 sn = f3(0.f);
    const uint32_t nb = vi_normal_buffer(vi);
    if (shading_normals && nb < s.vbuf_count) {
        const uint8_t* nbuf = s.vbufs[nb];
        const uint32_t no = vi_normal_offset(vi), ns = vi_normal_stride(vi);
        const float3 n0 = load_f3(nbuf, no, ns, tri.x), n1 = load_f3(nbuf, no, ns, tri.y), n2 = load_f3(nbuf, no, ns, tri.z);
        sn = n0 + (n1 - n0) * b1 + (n2 - n0) * b2;
        valid = !((sn.x == 0.f && sn.y == 0.f && sn.z == 0.f) || any_nan(sn));
    }
    if (!valid) {
        r.ns = r.ng;
        r.tg = pack_normal(normalize_rn(dPdu));
    } else {
        sn = normalize(xform_vector(M, sn));
        r.ns = pack_normal(sn);
        r.tg = pack_normal(normalize(dPdu - sn * dot(sn, dPdu)));
        if (dot(sn, gn) < 0.f) r.ng = pack_normal(-gn);
    }
}

S2D void shading_finish(const DevScene& s, uint32_t inst, float3 v0, float3 e1, float3 e2, float b1, float b2, SD& r) {
    r.pos = xform_point(s.transforms + 3 * (size_t)inst, v0 + e1 * b1 + e2 * b2);
    r.n = unpack_normal(r.ns);
    r.t = unpack_normal(r.tg);
    r.b = cross(r.n, r.t);
    r.gn = unpack_normal(r.ng);
}

S2D SD make_shading(const DevScene& s, uint32_t inst, uint32_t prim, float b1, float b2, bool shading_normals) {
    SD r;
    float3 v0, e1, e2;
    shading_terms(s, inst, prim, b1, b2, shading_normals, r, v0, e1, e2);
    shading_finish(s, inst, v0, e1, e2, b1, b2, r);
    return r;
}

// Baked shading record of a BVH triangle whose instance's vertex data has neither texture
// coordinates nor normals (the benchmark meshes): makeTriangleShadingData then depends only on the
// object-space vertices, the instance transform and the barycentrics, and every term but the hit
// position is a property of the triangle.  k_bake_shading evaluates shading_terms once per triangle
// and keeps {v0, material address}, {v1 - v0, area}, {v2 - v0, packed geometric normal},
// {packed tangent, 1 (valid), 0, 0}; a hit then reads this 64-byte record and the transform (two
// independent loads after the triangle record) instead of the chain instance -> vertex info ->
// indices -> positions.  The terms are explicitly rounded and the record and gather paths share
// one shading_finish, so the results are identical.
constexpr uint32_t kShadeRecValid = 1u;
S2D SD make_shading_rec(const DevScene& s, uint32_t tri, uint32_t inst, uint32_t prim, float b1, float b2,
                        bool shading_normals) {
    SD r;
    float3 v0, e1, e2;
    bool baked = false;
    if (s.shade_recs) {
        const float4* rp = s.shade_recs + 4 * (size_t)tri;
        const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1), r2 = __ldg(rp + 2), r3 = __ldg(rp + 3);
        if (__float_as_uint(r3.y) == kShadeRecValid) {
            v0 = f3(r0.x, r0.y, r0.z); e1 = f3(r1.x, r1.y, r1.z); e2 = f3(r2.x, r2.y, r2.z);
            r.mat = __float_as_uint(r0.w);
            r.area = r1.w;
            r.ng = __float_as_uint(r2.w);
            r.ns = r.ng;
            r.tg = __float_as_uint(r3.x);
            r.uv = make_float2(0.f, 0.f);
            baked = true;
        }
    }
    if (!baked) shading_terms(s, inst, prim, b1, b2, shading_normals, r, v0, e1, e2);
    shading_finish(s, inst, v0, e1, e2, b1, b2, r);
    return r;
}

// ApplyNormalMap (material.hlsli:78-105, gNormalMaps): the bump image (index, strength and
// channel count at bytes 36..47 of the material record) perturbs the shading normal in the
// tangent frame; normal and tangent are re-packed octahedrally as the reference stores them.
// The bitangent sign is +1: the reference never sets SHADING_FLAG_FLIP_BITANGENT.
S2D void apply_normal_map(const DevScene& s, SD& sd) {
    const uint8_t* rec = s.material_data + sd.mat + 36;
    const uint32_t img = ld_u32(rec, 0), channels = ld_u32(rec, 8);
    const float scale = ld_f32(rec, 4);
    if (img >= s.image_count || !(scale > 0.f)) return;
    const float4 t = sample_image(s.images[img], sd.uv);
    float3 bump = channels == 2 ? f3(t.x, t.y, 1.f) : f3(t.x, t.y, t.z);
    bump.x = (bump.x * 2.f - 1.f) * scale;
    bump.y = -(bump.y * 2.f - 1.f) * scale;
    const float3 n = normalize(sd.t * bump.x + cross(sd.n, sd.t) * bump.y + sd.n * bump.z);
    const float3 tg = normalize(sd.t - n * dot(n, sd.t));
    sd.ns = pack_normal(n);
    sd.tg = pack_normal(tg);
    sd.n = unpack_normal(sd.ns);
    sd.t = unpack_normal(sd.tg);
    sd.b = cross(sd.n, sd.t);
}

// makeTriangleShadingData from an object-space position (shading_data.hlsli:153-173): the
// barycentrics are recovered from the position (used for vertices stored in the hash grid).
S2D SD make_shading_local(const DevScene& s, uint32_t inst, uint32_t prim, float3 lp, bool shading_normals) {
    const uint2 id = s.instances[inst];
    const VInfo vi = load_vinfo(s, id.y & 0xffffu);
    const uint3 tri = load_triangle_indices(s.vbufs[vi_index_buffer(vi)], vi_index_offset(vi), vi_index_stride(vi), prim);
    const uint8_t* pb = s.vbufs[vi_position_buffer(vi)];
    const uint32_t po = vi_position_offset(vi), ps = vi_position_stride(vi);
    const float3 v0 = load_f3(pb, po, ps, tri.x), v1 = load_f3(pb, po, ps, tri.y), v2 = load_f3(pb, po, ps, tri.z);
    const float3 e1 = v1 - v0, e2 = v2 - v0, pv = lp - v0;
    const float d00 = dot(e1, e1), d01 = dot(e1, e2), d11 = dot(e2, e2), d20 = dot(pv, e1), d21 = dot(pv, e2);
    const float den = d00 * d11 - d01 * d01;
    const float b1 = (d11 * d20 - d01 * d21) / den, b2 = (d00 * d21 - d01 * d20) / den;
    SD r = make_shading(s, inst, prim, b1, b2, shading_normals);
    r.pos = xform_point(s.transforms + 3 * (size_t)inst, lp);
    return r;
}
