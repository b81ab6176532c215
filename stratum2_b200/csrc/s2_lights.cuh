// Light sampling (src/Shaders/common/lights.hlsli): uniform light instance -> uniform primitive ->
// uniform area for emissive triangles, and hierarchical importance sampling of the environment map
// over its luminance mip pyramid.
#pragma once
#include "s2_bsdf.cuh"

// Texels outside the level read as 0.  (The reference's descent can address one column or row
// past a level after skipping an all-black level; those reads are undefined there.)
S2D float texel_lum(const DevImage& im, uint32_t level, int x, int y) {
    if (x < 0 || y < 0 || x >= (int)im.lw[level] || y >= (int)im.lh[level]) return 0.f;
    return im.lum[im.lum_offset[level] + (size_t)y * im.lw[level] + x];
}

// SampleTexel (lights.hlsli:49-96), at most 10 levels.  With the precomputed block table each
// level is one 16-byte load instead of four texel loads and two sines.
S2D float2 sample_texel(const DevImage& im, float rx, float ry, float& pdf) {
    const uint32_t levels = im.levels;
    pdf = 1.f;
    int cx = 0, cy = 0;
    uint32_t lx = 1, ly = 1;
    const uint32_t lim = min(11u, levels - 1);
    for (uint32_t i = 1; i < lim; ++i) {
        const uint32_t level = levels - 1 - i;
        const uint32_t ex = im.lw[level], ey = im.lh[level];
        cx *= (int)(ex / lx);
        cy *= (int)(ey / ly);
        float p[4] = {0.f, 0.f, 0.f, 0.f};
        if (im.nested) {
            // all-zero weights outside the level, as the per-texel path computes
            if (cx >= (int)ex || cy >= (int)ey || (cx & 1) || (cy & 1)) continue;
            const float4 q = __ldg(im.quad + im.quad_offset[level] + (size_t)(cy >> 1) * im.qw[level] + (cx >> 1));
            if (q.x < 0.f) continue;
            p[0] = q.x; p[1] = q.y; p[2] = q.z; p[3] = q.w;
            for (int j = 0; j < 4; ++j) {
                if (j == 3 || rx < p[j]) {
                    cx += j % 2; cy += j / 2; pdf *= p[j]; rx /= p[j];
                    break;
                }
                rx -= p[j];
            }
            lx = ex; ly = ey;
            continue;
        }
        const float inv_h = 1.f / (float)ey;
        if ((int)ex - cx > 1) {
            const float sy = sinf(S2_PI * (cy + 0.5f) * inv_h);
            p[0] = texel_lum(im, level, cx, cy) * sy;
            p[1] = texel_lum(im, level, cx + 1, cy) * sy;
        }
        if ((int)ey - cy > 1) {
            const float sy = sinf(S2_PI * (cy + 1.5f) * inv_h);
            p[2] = texel_lum(im, level, cx, cy + 1) * sy;
            p[3] = texel_lum(im, level, cx + 1, cy + 1) * sy;
        }
        const float sum = p[0] + p[1] + p[2] + p[3];
        if (sum < 1e-6f) continue;
        for (int j = 0; j < 4; ++j) p[j] /= sum;
        for (int j = 0; j < 4; ++j) {
            if (j == 3 || rx < p[j]) {
                cx += j % 2; cy += j / 2; pdf *= p[j]; rx /= p[j];
                break;
            }
            rx -= p[j];
        }
        lx = ex; ly = ey;
    }
    pdf *= (float)(lx * ly);
    return make_float2(((float)cx + rx) / (float)lx, ((float)cy + ry) / (float)ly);
}

// SampleTexelPdf (lights.hlsli:97-138); one table load when the mip levels nest
S2D float sample_texel_pdf(const DevImage& im, float2 uv) {
    const uint32_t levels = im.levels;
    if (im.nested) {
        const uint32_t f = im.pdf_level;
        const int ux = (int)((float)im.lw[f] * uv.x), uy = (int)((float)im.lh[f] * uv.y);
        if (ux >= 0 && uy >= 0 && ux < (int)im.lw[f] && uy < (int)im.lh[f])
            return __ldg(im.pdf + (size_t)uy * im.lw[f] + ux);
    }
    float pdf = 1.f;
    uint32_t lx = 1, ly = 1;
    const uint32_t lim = min(11u, levels - 1);
    for (uint32_t i = 1; i < lim; ++i) {
        const uint32_t level = levels - 1 - i;
        const uint32_t ex = im.lw[level], ey = im.lh[level];
        const float inv_h = 1.f / (float)ey;
        const int ux = (int)((float)ex * uv.x), uy = (int)((float)ey * uv.y);
        const int cx = (ux / 2) * 2, cy = (uy / 2) * 2;
        const int ox = min(ux - cx, 1), oy = min(uy - cy, 1);
        float p[4] = {0.f, 0.f, 0.f, 0.f};
        if ((int)ex - cx > 1) {
            const float sy = sinf(S2_PI * (cy + 0.5f) * inv_h);
            p[0] = texel_lum(im, level, cx, cy) * sy;
            p[1] = texel_lum(im, level, cx + 1, cy) * sy;
        }
        if ((int)ey - cy > 1) {
            const float sy = sinf(S2_PI * (cy + 1.5f) * inv_h);
            p[2] = texel_lum(im, level, cx, cy + 1) * sy;
            p[3] = texel_lum(im, level, cx + 1, cy + 1) * sy;
        }
        const float sum = p[0] + p[1] + p[2] + p[3];
        if (sum < 1e-6f) continue;
        pdf *= p[oy * 2 + ox] / sum;
        lx = ex; ly = ey;
    }
    return pdf * (float)(lx * ly);
}

S2D bool has_env(const DevScene& s) { return s.env_address != 0xffffffffu; }

// The descriptor whose luminance tables drive environment sampling and its pdf: the environment
// image's own, or with S2_FLAG_ENV_FOOTPRINT_PDF the bilinear-footprint tables.
S2D const DevImage& env_sampling_image(const DevScene& s, uint32_t img) {
    return (s.env_fp_on && s.env_fp) ? *s.env_fp : s.images[img];
}

// EvaluateEnvironment (lights.hlsli:143-164): emission and its solid-angle pdf
S2D float3 eval_env(const DevScene& s, float3 dir, float& pdfw) {
    pdfw = 0.f;
    if (!has_env(s)) return f3(0.f);
    const float4 rec = *(const float4*)(s.material_data + s.env_address);
    float3 e = f3(rec.x, rec.y, rec.z);
    const uint32_t img = __float_as_uint(rec.w);
    if (img < s.image_count) {
        const float2 uv = cartesian_to_spherical_uv(dir);
        const float4 t = sample_image(s.images[img], uv);
        e = e * f3(t.x, t.y, t.z);
        pdfw = sample_texel_pdf(env_sampling_image(s, img), uv) / (2.f * S2_PI * S2_PI * sqrtf(1.f - dir.y * dir.y));
    } else {
        pdfw = 1.f / (4.f * S2_PI);
    }
    if (s.light_count > 0) pdfw *= s.env_sample_prob;
    return e;
}

struct Illum {
    float3 radiance;
    float pdf;          // area measure for triangle lights, solid angle for the environment
    float3 dir;         // direction to the light
    float dist;
    float cos_light;
    bool finite;
};

// SampleEmission + SampleIllumination (lights.hlsli:166-262).  The environment branch returns the
// sampled direction (the reference leaves mDirectionToLight unset there).
S2D Illum sample_illum(const DevScene& s, float4 rnd, float3 ref, bool shading_normals) {
    Illum r;
    r.radiance = f3(0.f); r.pdf = 0.f; r.dir = f3(0.f); r.dist = 0.f; r.cos_light = 0.f; r.finite = true;
    const uint32_t L = s.light_count;
    const float envp = s.env_sample_prob;
    if (has_env(s)) {
        if (L == 0 || rnd.w < envp) {
            const uint32_t img = ld_u32(s.material_data, s.env_address + 12);
            float3 dir;
            float pdf;
            if (img < s.image_count) {
                const float2 uv = sample_texel(env_sampling_image(s, img), rnd.x, rnd.y, pdf);
                dir = spherical_uv_to_cartesian(uv);
                pdf /= (2.f * S2_PI * S2_PI * sqrtf(1.f - pow2(dir.y)));
            } else {
                dir = sample_uniform_sphere(rnd.x, rnd.y);
                pdf = 1.f / (4.f * S2_PI);
            }
            if (L > 0) pdf *= envp;
            r.pdf = pdf; r.finite = false; r.dist = S2_INF; r.cos_light = 1.f; r.dir = dir;
            float tmp;
            r.radiance = eval_env(s, dir, tmp);
            return r;
        }
        if (L > 0) rnd.w = (rnd.w - envp) / (1.f - envp);
    }
    if (L == 0) return r;
    uint32_t light;
    float pdf;
    if (s.light_power_pick) {  // alias table: one uniform number picks a column and its threshold
        const float u = rnd.z * (float)L;
        const uint32_t col = min((uint32_t)u, L - 1u);
        const float2 a = s.light_alias[col];
        light = (u - (float)col) < a.x ? col : __float_as_uint(a.y);
        pdf = s.light_pick_pdf[light];
        const uint2 range = s.light_tri_range[light];
        const uint32_t prim = (uint32_t)(rnd.w * range.y) % max(range.y, 1u);
        const float4* lt = s.light_tris + 4 * (size_t)(range.x + prim);
        const float4 t0 = lt[0];
        if (t0.w > 0.f) {  // baked triangle: one 64-byte record instead of make_shading's gathers
            const float4 t1 = lt[1], t2 = lt[2], t3 = lt[3];
            const float2 b = sample_uniform_triangle(rnd.x, rnd.y);
            const float3 pos = f3(t0.x + t1.x * b.x + t2.x * b.y, t0.y + t1.y * b.x + t2.y * b.y, t0.z + t1.z * b.x + t2.z * b.y);
            if (has_env(s)) pdf *= 1.f - envp;
            r.radiance = f3(t1.w, t2.w, t3.w);
            r.dir = pos - ref;
            r.dist = length(r.dir);
            r.dir = r.dir / r.dist;
            r.cos_light = -dot(f3(t3.x, t3.y, t3.z), r.dir);
            r.pdf = pdf / ((float)range.y * t0.w);
            if (r.cos_light <= 0.f) { r.radiance = f3(0.f); r.pdf = 0.f; }
            return r;
        }
    } else {
        light = (uint32_t)(rnd.z * L) % L;
        pdf = 1.f / (float)L;
    }
    const uint32_t inst = s.light_instance_map[light];
    if (has_env(s)) pdf *= 1.f - envp;
    if ((s.instances[inst].x & 0xfu) != 0u) return r;
    const uint32_t pc = s.prim_counts[inst];
    const uint32_t prim = (uint32_t)(rnd.w * pc) % pc;
    pdf /= (float)pc;
    const float2 b = sample_uniform_triangle(rnd.x, rnd.y);
    const SD sd = make_shading(s, inst, prim, b.x, b.y, shading_normals);
    pdf /= sd.area;
    const Mat m = load_material(s, sd.mat, sd.uv);
    r.radiance = m.emission();
    r.dir = sd.pos - ref;
    r.dist = length(r.dir);
    r.dir = r.dir / r.dist;
    r.cos_light = -dot(sd.gn, r.dir);
    r.pdf = pdf;
    if (r.cos_light <= 0.f) { r.radiance = f3(0.f); r.pdf = 0.f; }  // one-sided lights
    return r;
}

// A point on a light to start a light subpath from (InitializeLightPath, testrenderer.slang:
// 983-1001): the light pick and triangle sampling of sample_illum, without its one-sidedness test
// against a reference point.  Area lights give the point, its geometric normal (the emitting side),
// the emission and the area pdf; the environment gives the direction toward it and its solid-angle
// pdf, from sample_illum's own environment branch.
struct LightPoint {
    float3 pos, n, radiance, dir;
    float pdf;
    bool finite, ok;
};
S2D LightPoint sample_light_point(const DevScene& s, float4 rnd, bool shading_normals) {
    LightPoint p;
    p.pos = p.n = p.radiance = p.dir = f3(0.f);
    p.pdf = 0.f; p.finite = true; p.ok = false;
    const uint32_t L = s.light_count;
    const float envp = s.env_sample_prob;
    if (has_env(s) && (L == 0 || rnd.w < envp)) {
        const Illum r = sample_illum(s, rnd, f3(0.f), shading_normals);
        p.finite = false; p.dir = r.dir; p.radiance = r.radiance; p.pdf = r.pdf;
        p.ok = r.pdf > 0.f && any_pos(r.radiance);
        return p;
    }
    if (L == 0) return p;
    if (has_env(s)) rnd.w = (rnd.w - envp) / (1.f - envp);
    uint32_t light;
    float pdf;
    if (s.light_power_pick) {
        const float u = rnd.z * (float)L;
        const uint32_t col = min((uint32_t)u, L - 1u);
        const float2 a = s.light_alias[col];
        light = (u - (float)col) < a.x ? col : __float_as_uint(a.y);
        pdf = s.light_pick_pdf[light];
    } else {
        light = (uint32_t)(rnd.z * L) % L;
        pdf = 1.f / (float)L;
    }
    if (has_env(s)) pdf *= 1.f - envp;
    const uint32_t inst = s.light_instance_map[light];
    if ((s.instances[inst].x & 0xfu) != 0u) return p;
    const uint32_t pc = s.prim_counts[inst];
    const uint32_t prim = (uint32_t)(rnd.w * pc) % pc;
    const float2 b = sample_uniform_triangle(rnd.x, rnd.y);
    const SD sd = make_shading(s, inst, prim, b.x, b.y, shading_normals);
    const Mat m = load_material(s, sd.mat, sd.uv);
    p.pos = sd.pos; p.n = sd.gn; p.radiance = m.emission();
    p.pdf = pdf / (float)pc / sd.area;
    p.ok = p.pdf > 0.f && any_pos(p.radiance);
    return p;
}

// IntersectionResult::LightSamplePdfA (lights.hlsli:264-272)
S2D float light_pdfa(const DevScene& s, uint32_t inst, float area) {
    if (s.light_count == 0) return 0.f;
    float pdf;
    if (s.light_power_pick) {  // instances outside the light list are never picked
        const uint32_t light = s.instance_light_map[inst];
        pdf = light < s.light_count ? s.light_pick_pdf[light] / ((float)s.prim_counts[inst] * area) : 0.f;
    } else {
        pdf = (1.f / (float)s.prim_counts[inst]) / (area * (float)s.light_count);
    }
    if (has_env(s)) pdf *= 1.f - s.env_sample_prob;
    return pdf;
}
