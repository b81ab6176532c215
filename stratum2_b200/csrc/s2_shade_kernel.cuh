// Shade kernel of the wavefront path tracer: the body of ProcessInteraction
// (src/Shaders/kernels/testrenderer.slang:816-935) with TraceRay's miss handling (:1026-1058),
// AddEmission (:788-808), ConnectToLight (:751-779; ReSTIR variant :665-683, :730-747) and
// StoreAuxillaryData (:195-218), plus the minPathLength gate of vcm.slang:922,960,977.
#pragma once
#include "s2_wavefront.cuh"

namespace s2 {

// Appends `want` lanes of the warp to a queue: one atomic per warp.  All 32 lanes must call.
S2D uint32_t warp_append(uint32_t* counter, bool want) {
    const uint32_t mask = __ballot_sync(0xffffffffu, want);
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t base = 0;
    if (mask) {
        const uint32_t leader = __ffs(mask) - 1;
        if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
        base = __shfl_sync(0xffffffffu, base, leader);
    }
    return base + __popc(mask & ((1u << lane) - 1u));
}

// The view a path belongs to, for its AOV writes: the single view of a wave render, or its entry
// in the batched view table (view index in meta bits 16..23; slot = pixel_offset + pixel).
struct AovTarget {
    const float* proj;
    const int* imin;
    const int* imax;
    const float* prev_inv;
    uint32_t width, pixel;
    float4* albedo;
    uint2* vis;
    float4* depth;
    float2* prev_uv;
    uint2* ids;
};
S2D AovTarget aov_target(const PTParams& P, uint32_t slot, uint32_t meta) {
    AovTarget t;
    if (P.views) {
        const ViewEntry& V = P.views[(meta >> 16) & 0xffu];
        t.proj = V.proj; t.imin = V.imin; t.imax = V.imax; t.prev_inv = V.prev_inv; t.width = V.width;
        t.pixel = slot - V.pixel_offset;
        t.albedo = V.aov_albedo; t.vis = V.aov_vis; t.depth = V.aov_depth; t.prev_uv = V.aov_prev_uv; t.ids = V.aov_ids;
    } else {
        t.proj = P.proj; t.imin = P.imin; t.imax = P.imax; t.prev_inv = P.prev_inv; t.width = P.width;
        t.pixel = slot % P.pixels;
        t.albedo = P.aov_albedo; t.vis = P.aov_vis; t.depth = P.aov_depth; t.prev_uv = P.aov_prev_uv; t.ids = P.aov_ids;
    }
    return t;
}

// A deferred shadow ray, or (direct) a contribution whose visibility is already known.
struct ShadowOut { float3 o, d, c; float tmax; bool valid, direct; };

// A light sample evaluated at one vertex: ReservoirSampleDataDI (testrenderer.slang:568-606).
struct DISample {
    float4 rnd;        // the sample (its four random numbers)
    float src_pdf;     // light-sampling pdf (area measure, or solid angle for the environment)
    float wtoa;        // cos_light / d^2 (1 for the environment)
    float mis;         // MIS weight against BSDF sampling
    float dist;
    float3 contrib;    // f * Le (shading-normal corrected)
    float3 dir;
    float vis;         // traced visibility (1 unless a reuse-visibility ray found the light occluded)
    S2D float target() const { return luminance(contrib) * wtoa; }
};

// traceVisibilityRay for a light sample, traced inline (S2_FLAG_RESTIR_REUSE_VISIBILITY).
S2D bool di_visible(const PTParams& P, const SD& sd, const DISample& c, uint2* vstack) {
    const SceneAlphaTest alpha{&P.scene, !(P.flags & S2F_NO_ALPHA)};
    TravHit h;
    TravCounters ctr{0, 0};
    if (!traverse<true, false>(make_trav_ray(ray_offset(sd.pos, sd.gn, c.dir), c.dir, 0.f), adjust_distance(c.dist),
                               P.scene.nodes, P.scene.tris, vstack, 128u, h, ctr, alpha))
        atomicOr(P.status, 1);
    atomicAdd(&P.stats[S_SHADOW], 1ull);
    return h.tri == 0xffffffffu;
}

template <bool LAMBERT>
S2D DISample eval_di(const DevScene& s, const Mat& m, const SD& sd, float3 in, float4 x, bool sn, float cp) {
    DISample c;
    c.rnd = x; c.contrib = f3(0.f); c.wtoa = 0.f; c.mis = 0.f; c.dist = 0.f; c.dir = f3(0.f); c.vis = 1.f;
    const Illum r = sample_illum(s, x, sd.pos, sn);
    c.src_pdf = r.pdf;
    if (luminance(r.radiance) > 0.f && r.pdf > 0.f) {
        const float3 out = sd.to_local(r.dir);
        float3 f; float fwd, rev;
        bsdf_eval<LAMBERT>(m, in, out, f, fwd, rev);
        f = f * sd.snc(in, out);
        fwd *= cp;
        c.contrib = f * r.radiance;
        c.wtoa = r.finite ? r.cos_light / pow2(r.dist) : 1.f;
        const float AtoW = r.finite ? pow2(r.dist) / r.cos_light : 1.f;
        c.mis = mis_w(r.pdf, fwd / AtoW);
        c.dist = r.dist;
        c.dir = r.dir;
    }
    return c;
}

// ReservoirReuse (testrenderer.slang:608-663): combines the current reservoir with a stored one
// (q) with pairwise power-heuristic MIS over the two domains' target pdfs.
template <bool LAMBERT>
S2D void reservoir_reuse(const PTParams& P, const Mat& m, const SD& sd, float3 in, float cp, const ReservoirRecord& q,
                         DISample& cur, float& iw, float& M, Rng& rng, bool sn, uint2* vstack) {
    const DevScene& s = P.scene;
    DISample nw = eval_di<LAMBERT>(s, m, sd, in, q.rnd, sn, cp);  // q's sample in the current domain
    // reuse visibility (testrenderer.slang:611-616): the reused sample's contribution carries its
    // visibility here, its target pdf stays unshadowed.  The reference also traces the current
    // sample's visibility in q's domain, but only that sample's target pdf is used there.
    if (vstack && nw.target() > 0.f && !di_visible(P, sd, nw, vstack)) nw.vis = 0.f;
    float phat_q = 0.f;                                                 // current sample in q's domain
    {
        SD sdq = make_shading_local(s, q.instance, q.primitive, q.local_pos, sn);
        if (!(P.flags & S2F_NO_NORMAL_MAPS)) apply_normal_map(s, sdq);
        const Mat mq = load_material(s, sdq.mat, sdq.uv);
        const float cpq = (P.flags & S2F_NO_RR) ? 1.f : cont_prob(mq);
        const DISample cq = eval_di<LAMBERT>(s, mq, sdq, q.local_dir_in, cur.rnd, sn, cpq);
        if (cq.target() > 0.f) phat_q = cq.target();
    }
    const float m0 = mis_w(M * cur.target(), q.M * phat_q);
    const float m1 = mis_w(q.M * q.target_pdf, M * nw.target());
    const float w0 = m0 * cur.target() * iw;
    const float w1 = m1 * nw.target() * q.W;
    M += q.M;
    const float total = w0 + w1;
    if (rng.next_float().x * total <= w1) cur = nw;
    iw = cur.target() > 0.f ? total / cur.target() : 0.f;
}

// Previous-frame camera-space position of world point pw (row-major 3x4 world-to-camera).
S2D float3 prev_camera_point(const float* pv, float3 pw) {
    return f3(pv[0] * pw.x + pv[1] * pw.y + pv[2] * pw.z + pv[3], pv[4] * pw.x + pv[5] * pw.y + pv[6] * pw.z + pv[7],
              pv[8] * pw.x + pv[9] * pw.y + pv[10] * pw.z + pv[11]);
}

// ViewData::toRaster (compat/scene.h:158-165), perspective projectPoint: raster position (pixels,
// image_min included) of camera-space point pc; leaves `out` unchanged and returns false when pc is
// behind the camera or outside the frustum.
S2D bool camera_to_raster(const float* proj, const int* imin, const int* imax, float3 pc, float2& out) {
    const float nr = proj[4];
    if (!((pc.z > 0.f) == (nr > 0.f) && pc.z != 0.f)) return false;
    const float x4 = pc.x * proj[0] + pc.z * proj[2], y4 = pc.y * proj[1] + pc.z * proj[3];
    const float z4 = fabsf(nr), w4 = pc.z * (nr > 0.f ? 1.f : -1.f);
    if (fabsf(x4) >= fabsf(w4) || fabsf(y4) >= fabsf(w4) || fabsf(z4) >= fabsf(w4)) return false;
    const float W = (float)(imax[0] - imin[0]), H = (float)(imax[1] - imin[1]);
    out = make_float2(imin[0] + W * (x4 / w4 * 0.5f + 0.5f), imin[1] + H * (-y4 / w4 * 0.5f + 0.5f));
    return true;
}

// One NEE connection: plain light sample, or RIS over restir_m candidates (+ hash-grid or
// screen-space reuse).
template <bool LAMBERT, bool RESTIR>
S2D ShadowOut connect_to_light(const PTParams& P, const Mat& m, const SD& sd, float3 in, float3 thr, Rng& rng, uint32_t len,
                               bool sn, uint32_t inst, uint32_t prim, const ViewEntry* V, uint32_t pixel, bool store_pixel,
                               uint2* vstack) {
    ShadowOut so;
    so.valid = false;
    so.direct = false;
    const DevScene& s = P.scene;
    const float cp = (P.flags & S2F_NO_RR) ? 1.f : cont_prob(m);
    float3 dir, contrib;
    float dist, w;
    if (RESTIR) {
        // SampleIlluminationReSTIR (testrenderer.slang:665-726)
        DISample best;
        best.rnd = make_float4(0.f, 0.f, 0.f, 0.f); best.contrib = f3(0.f); best.wtoa = 0.f; best.mis = 0.f;
        best.dist = 0.f; best.dir = f3(0.f); best.src_pdf = 0.f;
        float wsum = 0.f;
        for (uint32_t i = 0; i < P.restir_m; ++i) {
            const DISample c = eval_di<LAMBERT>(s, m, sd, in, rng.next_float(), sn, cp);
            const float target = c.target();
            if (target <= 0.f) continue;
            const float risw = target / c.src_pdf;
            wsum += risw;
            if (rng.next_float().x <= risw / wsum) best = c;
        }
        float iw = best.target() > 0.f ? wsum / ((float)P.restir_m * best.target()) : 0.f;
        // gReSTIR_DI_Reuse_Visibility (testrenderer.slang:689-694): the canonical sample's visibility
        // before reuse; an occluded one gets W = 0
        // screen-space reuse at the primary vertex of an image path; V: its view in a batched call
        const bool ss_here = P.ss_on && len == 1 && (!P.views || V != nullptr);
        uint2* vs = (vstack && (P.reuse || ss_here)) ? vstack : nullptr;
        if (vs) {
            if (best.target() > 0.f && !di_visible(P, sd, best, vs)) best.vis = 0.f;
            if (!(best.vis > 0.f)) iw = 0.f;
        }
        if (ss_here) {
            // screen-space reuse at the primary vertex: the previous call's reservoirs at the
            // reprojected pixel and at ss_spatial random pixels within ss_radius of it, each
            // combined with the running reservoir by ReservoirReuse's two-domain resampling.  A
            // batched call keeps one reservoir per pixel of every view, views at their pixel offsets.
            const float* vproj = V ? V->proj : P.proj;
            const int* vimin = V ? V->imin : P.imin;
            const int* vimax = V ? V->imax : P.imax;
            const uint32_t vw = V ? V->width : P.width, vh = V ? V->height : P.height;
            const uint32_t base = V ? V->pixel_offset : 0u;
            float M = (float)P.restir_m;
            float2 pr;
            if (P.ss_prev_valid &&
                camera_to_raster(vproj, vimin, vimax,
                                 prev_camera_point(V ? V->prev_inv : P.prev_inv,
                                                   xform_point(s.motion_transforms + 3 * (size_t)inst, sd.pos)), pr)) {
                for (uint32_t j = 0; j <= P.ss_spatial; ++j) {
                    float2 q = pr;
                    if (j > 0) {
                        const float4 u = rng.next_float();
                        const float2 d = sample_concentric_disc(u.x, u.y);
                        q = make_float2(pr.x + d.x * P.ss_radius, pr.y + d.y * P.ss_radius);
                    }
                    const float fx = floorf(q.x - (float)vimin[0]), fy = floorf(q.y - (float)vimin[1]);
                    if (!(fx >= 0.f && fy >= 0.f && fx < (float)vw && fy < (float)vh)) continue;
                    const ReservoirRecord rq = P.ss_prev[base + (uint32_t)fy * vw + (uint32_t)fx];
                    if (!(rq.W > 0.f)) continue;
                    reservoir_reuse<LAMBERT>(P, m, sd, in, cp, rq, best, iw, M, rng, sn, vs);
                }
            }
            if (store_pixel) {
                ReservoirRecord rec;
                rec.local_pos = xform_point(s.inv_transforms + 3 * (size_t)inst, sd.pos);
                rec.instance = inst;
                rec.primitive = prim;
                rec.rnd = best.rnd;
                rec.target_pdf = best.target();
                rec.W = iw > 0.f ? iw : 0.f;
                rec.M = fminf(M, P.max_m * (float)P.restir_m);
                rec.local_dir_in = in;
                rec.pad = 0.f;
                P.ss_cur[base + pixel] = rec;
            }
        }
        if (P.reuse) {
            float M = (float)P.restir_m;
            if (P.prev_valid) {
                const float4 dr = rng.next_float();
                const float2 disc = sample_concentric_disc(dr.x, dr.y);
                const float csz = hg_cell_size(P.grid_prev, sd.pos);
                const float3 qp = sd.pos + sd.to_world(f3(disc.x * csz, disc.y * csz, 0.f));
                const uint32_t cell = hg_find_cell<false>(P.grid_prev, qp, hg_cell_size(P.grid_prev, qp));
                if (cell != 0xffffffffu) {
                    const uint32_t count = P.grid_prev.cell_counters[cell];
                    if (count > 0) {
                        const uint32_t off = P.grid_prev.indices[cell];
                        const uint32_t k = rng.next().x % count;
                        const ReservoirRecord q = P.grid_prev.data[P.grid_prev.data_indices[off + k]];
                        reservoir_reuse<LAMBERT>(P, m, sd, in, cp, q, best, iw, M, rng, sn, vs);
                    }
                }
            }
            if (iw > 0.f) {
                ReservoirRecord rec;
                rec.local_pos = xform_point(s.inv_transforms + 3 * (size_t)inst, sd.pos);
                rec.instance = inst;
                rec.primitive = prim;
                rec.rnd = best.rnd;
                rec.target_pdf = best.target();
                rec.W = iw;
                rec.M = fminf(M, P.max_m * (float)P.restir_m);
                rec.local_dir_in = in;
                rec.pad = 0.f;
                hg_append(P.grid_cur, sd.pos, rec);
            }
        }
        if (!(iw > 0.f)) return so;
        iw *= best.wtoa;  // 1/pdfA -> 1/pdfW
        contrib = thr * best.contrib * (iw * best.vis);
        so.direct = vs != nullptr;  // visibility already traced: AddRadiance without a shadow ray (:742-743)
        w = best.mis;
        dir = best.dir;
        dist = best.dist;
    } else {
        if (len + 1 < P.min_len) {  // shorter than minPathLength: advance the stream by one draw only
            rng.skip();
            return so;
        }
        const float4 x = rng.next_float();
        const Illum r = sample_illum(s, x, sd.pos, sn);
        if (all_nonpos(r.radiance) || r.pdf <= 0.f) return so;
        const float AtoW = r.finite ? pow2(r.dist) / r.cos_light : 1.f;
        const float dpw = r.pdf * AtoW;
        const float3 out = sd.to_local(r.dir);
        float3 f; float fwd, rev;
        bsdf_eval<LAMBERT>(m, in, out, f, fwd, rev);
        f = f * sd.snc(in, out);
        fwd *= cp;
        contrib = thr * r.radiance * f / dpw;
        w = mis_w(r.pdf, fwd / AtoW);
        dir = r.dir;
        dist = r.dist;
    }
    if (!(w > 0.f) || all_nonpos(contrib)) return so;
    if (len + 1 < P.min_len) return so;
    so.o = ray_offset(sd.pos, sd.gn, dir);
    so.d = dir;
    so.tmax = adjust_distance(dist);
    so.c = f3(fmaxf(contrib.x * w, 0.f), fmaxf(contrib.y * w, 0.f), fmaxf(contrib.z * w, 0.f));
    so.valid = true;
    return so;
}

// Resident 128-thread blocks per SM the shade variants are compiled for: the plain NEE variants at
// 64 registers (8 blocks; measured 2-3 % faster on B200 than 128 registers and 4 blocks despite
// the spills); the ReSTIR and radiance-cache variants, which need more live state, at 3 blocks
// (up to 170 registers).
template <bool RESTIR, bool CACHE> constexpr int kShadeMinBlocks = (RESTIR || CACHE) ? 3 : 8;

template <bool LAMBERT, bool RESTIR, bool CACHE = false>
__global__ void __launch_bounds__(128, kShadeMinBlocks<RESTIR, CACHE>) k_shade(PTParams P, uint32_t parity) {
    // traversal stacks of the inline reuse-visibility rays (ReSTIR variants only)
    __shared__ uint2 vstack[RESTIR ? S2_STACK_SMEM * 128 : 1];
    const uint32_t count = P.counters[parity];
    const PathQueue qi = P.q[parity];
    const PathQueue qo = P.q[1 - parity];
    const DevScene& s = P.scene;
    const bool nee = !(P.flags & S2F_NO_NEE);
    const bool sn = !(P.flags & S2F_NO_SN);
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t rounded = (count + 31u) & ~31u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rounded; i += stride) {
        bool alive = false, shadow = false, cq = false, tr = false;
        float4 n0, n1, n2;
        uint4 n3;
        float4 c_pos, c_thr, c_rad;
        ShadowOut so;
        so.valid = false;
        uint32_t slot = 0;
        if (i < count) {
            const uint32_t pi = P.sort_on ? P.sort_perm[i] : i;  // material-sorted order
            const float4 a = qi.s0[pi], b = qi.s1[pi], c = qi.s2[pi];
            const uint4 rs = qi.s3[pi];
            const float4 h = P.hits[pi];
            float3 org = f3(a.x, a.y, a.z);
            float dir_pdf = a.w;
            const float3 dir = f3(b.x, b.y, b.z);
            float3 thr = f3(b.w, c.x, c.y);
            slot = __float_as_uint(c.z);
            const uint32_t meta = __float_as_uint(c.w);
            const uint32_t len = (meta & 0xffu) + 1u;  // TraceRay: mPathLength++
            const bool aov = (meta & 0x100u) && len == 1;
            Rng rng;
            rng.px = rs.x; rng.py = rs.y; rng.seed = rs.z; rng.ctr = rs.w; rng.pcg32 = (P.flags & S2F_PCG32) != 0;
            const uint32_t tri = __float_as_uint(h.y);
            if (tri == 0xffffffffu) {
                // ---- miss: environment emission (TraceRay, testrenderer.slang:1036-1054)
                if (aov) {
                    const AovTarget A = aov_target(P, slot, meta);
                    const uint32_t pix = A.pixel;
                    if (A.albedo) A.albedo[pix] = make_float4(1.f, 1.f, 1.f, 1.f);
                    if (A.vis) A.vis[pix] = make_uint2(0xffffffffu, pack_normal(dir));
                    if (A.depth) A.depth[pix] = make_float4(S2_INF, S2_INF, 1.f, 1.f);
                    if (A.prev_uv) {
                        const uint32_t px = pix % A.width, py = pix / A.width;
                        A.prev_uv[pix] = make_float2(((float)px + 0.5f) / (float)(A.imax[0] - A.imin[0]),
                                                     ((float)py + 0.5f) / (float)(A.imax[1] - A.imin[1]));
                    }
                    if (A.ids) A.ids[pix] = make_uint2(0xffffffffu, 0xffffffffu);
                }
                float env_pdf = 0.f;
                const float3 e = len >= P.min_len ? thr * eval_env(s, dir, env_pdf) : f3(0.f);
                if (any_pos(e)) {
                    float w = 1.f;
                    if (len > 1 && nee && dir_pdf > 0.f) {
                        const float lp = (P.flags & S2F_REF_ENV_MIS) ? (S2_INV_PI / pow2(s.scene_sphere.w)) : env_pdf;
                        w = mis_w(dir_pdf, lp);
                    }
                    if (w > 0.f) add_contrib(P, slot, e * w);
                }
            } else {
                const float4 tr0 = s.tris[3 * (size_t)tri], tr1 = s.tris[3 * (size_t)tri + 1];
                const uint32_t inst = __float_as_uint(tr0.w), prim = __float_as_uint(tr1.w);
                SD sd = make_shading_rec(s, tri, inst, prim, h.z, h.w, sn);
                if (!(P.flags & S2F_NO_NORMAL_MAPS)) apply_normal_map(s, sd);
                const float isect_dist = half_round(h.x);
                const float isect_pdfa = half_round(light_pdfa(s, inst, sd.area));
                Mat m = load_material(s, sd.mat, sd.uv);
                // cache-form path regularisation: after the first bounce every vertex is at least
                // cache_rough rough
                if (CACHE && P.cache_on && P.cache_rough > 0.f && len >= 2) {
                    const uint32_t floor8 = pk8(P.cache_rough);
                    if (((m.w[2] >> 8) & 0xffu) < floor8) m.w[2] = (m.w[2] & ~0xff00u) | (floor8 << 8);
                }
                const float3 in = sd.to_local(-dir);
                const float cos_in = fabsf(in.z);
                if (aov) {
                    // StoreAuxillaryData (testrenderer.slang:195-218)
                    const AovTarget A = aov_target(P, slot, meta);
                    const uint32_t pix = A.pixel;
                    const float3 bc = m.base();
                    if (A.albedo) A.albedo[pix] = make_float4(bc.x, bc.y, bc.z, 1.f);
                    if (A.vis) A.vis[pix] = make_uint2((inst & 0xffffu) | (prim << 16), sd.ns);
                    if (A.ids) A.ids[pix] = make_uint2(inst, prim);
                    const float3 pw = xform_point(s.motion_transforms + 3 * (size_t)inst, sd.pos);
                    const float3 pc = prev_camera_point(A.prev_inv, pw);
                    const uint32_t px = pix % A.width, py = pix / A.width;
                    const float W = (float)(A.imax[0] - A.imin[0]), H = (float)(A.imax[1] - A.imin[1]);
                    float2 pr = make_float2((float)px + 0.5f, (float)py + 0.5f);
                    camera_to_raster(A.proj, A.imin, A.imax, pc, pr);
                    if (A.prev_uv) A.prev_uv[pix] = make_float2(pr.x / W, pr.y / H);
                    if (A.depth) A.depth[pix] = make_float4(isect_dist, length(pc), 1.f, 1.f);
                }
                // ---- emission (surface lights are one-sided)
                if (in.z > 0.f) {
                    const float3 e = thr * m.emission();
                    if (any_pos(e) && len >= P.min_len) {
                        float w = 1.f;
                        if (len > 1 && nee && dir_pdf > 0.f) w = mis_w(dir_pdf * (cos_in / pow2(isect_dist)), isect_pdfa);
                        if (w > 0.f) add_contrib(P, slot, e * w);
                    }
                }
                // ---- learned radiance cache: the terminal vertex of a non-training path takes its
                // scattered radiance from the cache; training paths record their vertices
                bool cached = false;
                if (CACHE && P.cache_on) {
                    const float4 pw = make_float4(sd.pos.x, sd.pos.y, sd.pos.z, __uint_as_float(slot));
                    if (!(meta & 0x200u)) {
                        if (len == P.cache_len) {
                            cached = true;
                            cq = any_pos(m.base());
                            c_pos = pw;
                            c_thr = make_float4(thr.x, thr.y, thr.z, 0.f);
                        }
                    } else if (len + 1 >= P.min_len && len < P.max_len) {
                        tr = true;
                        c_pos = pw;
                        c_thr = make_float4(thr.x, thr.y, thr.z, 0.f);
                        c_rad = P.accum[slot & ~kTrainSlot];
                    }
                }
                if (!cached && len < P.max_len && any_pos(m.base())) {
                    const bool sing = mat_singular<LAMBERT>(m);
                    // the path's view and pixel within it (batched training paths have neither)
                    const ViewEntry* sview = (P.views && !(slot & kTrainSlot)) ? &P.views[(meta >> 16) & 0xffu] : nullptr;
                    const uint32_t spix = sview ? slot - sview->pixel_offset : slot % P.pixels;
                    if (!sing && nee)
                        so = connect_to_light<LAMBERT, RESTIR>(P, m, sd, in, thr, rng, len, sn, inst, prim, sview, spix, aov,
                                                               (RESTIR && (P.flags & S2F_REUSE_VIS)) ? vstack + threadIdx.x : nullptr);
                    const float cp = fminf(1.f, cont_prob(m));
                    bool cont = true;
                    if (!(P.flags & S2F_NO_RR)) {
                        const float4 u = rng.next_float();
                        if (u.x > cp) cont = false;
                    }
                    if (cont) {
                        const float4 rnd = rng.next_float();
                        float3 sdir, refl;
                        float fwd, rev, rough;
                        bsdf_sample<LAMBERT>(m, in, rnd, sdir, refl, fwd, rev, rough);
                        const float cpm = (P.flags & S2F_NO_RR) ? 1.f : cp;
                        fwd *= cpm;
                        thr = thr * refl / fwd;
                        dir_pdf = (rough == 0.f || sing) ? 0.f : half_round(fwd);
                        thr = thr * sd.snc(in, sdir);
                        const float3 wd = sd.to_world(sdir);
                        const float3 nd = unpack_normal(pack_normal(wd));
                        org = ray_offset(sd.pos, sd.gn, wd);
                        if (any_nan(thr)) {
                            atomicAdd(&P.stats[S_NAN], 1ull);
                        } else if (any_pos(thr)) {
                            alive = true;
                            n0 = make_float4(org.x, org.y, org.z, dir_pdf);
                            n1 = make_float4(nd.x, nd.y, nd.z, thr.x);
                            n2 = make_float4(thr.y, thr.z, __uint_as_float(slot),
                                             __uint_as_float((meta & ~0xffu) | len));
                            n3 = make_uint4(rng.px, rng.py, rng.seed, rng.ctr);
                        }
                    }
                }
            }
            if (so.valid && so.direct) {
                add_contrib(P, slot, so.c);
                so.valid = false;
            }
            shadow = so.valid;
        }
        const uint32_t qi_out = warp_append(&P.counters[1 - parity], alive);
        if (alive) {
            qo.s0[qi_out] = n0; qo.s1[qi_out] = n1; qo.s2[qi_out] = n2; qo.s3[qi_out] = n3;
            if (P.ray_sort_on) P.sort_keys[qi_out] = ray_key(s, f3(n0.x, n0.y, n0.z), f3(n1.x, n1.y, n1.z));
        }
        const uint32_t si = warp_append(&P.counters[sh_counter(P)], shadow);
        if (shadow) {
            P.sh_o[si] = make_float4(so.o.x, so.o.y, so.o.z, so.tmax);
            P.sh_d[si] = make_float4(so.d.x, so.d.y, so.d.z, __uint_as_float(slot));
            P.sh_c[si] = make_float4(so.c.x, so.c.y, so.c.z, 0.f);
        }
        if (CACHE && P.cache_on) {
            const uint32_t ci = warp_append(&P.counters[C_CACHEQ], cq);
            if (cq && ci < P.cq_cap) { P.cq_pos[ci] = c_pos; P.cq_thr[ci] = c_thr; }
            const uint32_t ti = warp_append(&P.counters[C_TRAIN], tr);
            if (tr && ti < P.tr_cap) { P.tr_pos[ti] = c_pos; P.tr_thr[ti] = c_thr; P.tr_rad[ti] = c_rad; }
        }
    }
}

}  // namespace s2
