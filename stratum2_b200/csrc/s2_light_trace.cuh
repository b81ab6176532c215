// Light tracing (TestRenderer's mLightTrace mode): light subpaths start at the lights
// (InitializeLightPath, testrenderer.slang:983-1020), every non-singular vertex connects to the
// pinhole camera (ConnectToCamera, :441-512) through a shadow ray whose contribution lands on the
// pixel it projects to, and the subpath continues by Russian roulette and BSDF sampling with the
// adjoint shading-normal correction (:886-933, shading_data.hlsli:35-55).  Traversal and occlusion
// reuse k_extend / k_occlude; the pixel contributions go to fixed-point totals (add_contrib with
// P.total_fx), so images do not depend on the order of the atomic additions.
#pragma once
#include "s2_shade_kernel.cuh"

namespace s2 {

// shadingNormalCorrection<Adjoint = true> (shading_data.hlsli:35-55)
S2D float snc_adjoint(const SD& sd, float3 in, float3 out) {
    const float3 lg = sd.to_local(sd.gn);
    const float a = dot(lg, in), c = dot(lg, out);
    if (sgnf(c) != sgnf(out.z) || sgnf(a) != sgnf(in.z)) return 0.f;  // light leak fix
    const float num = c * in.z, den = out.z * a;
    return fabsf(den) > 1e-5f ? fabsf(num / den) : 1.f;
}

// One light subpath per work item, appended densely to queue 0.
__global__ void __launch_bounds__(256) k_light_gen(PTParams P, uint32_t sample) {
    const DevScene& s = P.scene;
    const bool sn = !(P.flags & S2F_NO_SN);
    const uint32_t n = P.lt_paths, rounded = (n + 31u) & ~31u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rounded; i += gridDim.x * blockDim.x) {
        bool ok = false;
        float3 org = f3(0.f), dir = f3(0.f), thr = f3(0.f);
        Rng rng;
        if (i < n) {
            // RandomSampler(seed, index, 0xFFFF) of the reference's light pass
            rng = make_rng(i, 0xFFFFu, P.frame_seed + sample, (P.flags & S2F_PCG32) != 0);
            const LightPoint lp = sample_light_point(s, rng.next_float(), sn);
            const float4 u = rng.next_float();
            if (lp.ok) {
                float3 t, b;
                if (lp.finite) {
                    // cosine-weighted emission about the emitting side: thr = Le / pdfA * pi
                    const float3 d = sample_cos_hemisphere(u.x, u.y);
                    make_orthonormal(lp.n, t, b);
                    dir = normalize(t * d.x + b * d.y + lp.n * d.z);
                    org = ray_offset(lp.pos, lp.n);
                    thr = lp.radiance * (S2_PI / lp.pdf);
                    ok = d.z > 0.f;
                } else {
                    // environment: parallel rays through a disc of the scene's bounding sphere; the
                    // disc's area (pi R^2) completes the throughput (the reference leaves it out)
                    const float2 xy = sample_concentric_disc(u.x, u.y);
                    make_orthonormal(-lp.dir, t, b);
                    const float R = s.scene_sphere.w;
                    const float3 c = f3(s.scene_sphere.x, s.scene_sphere.y, s.scene_sphere.z);
                    org = c + (t * xy.x + b * xy.y + lp.dir) * R;
                    dir = -lp.dir;
                    thr = lp.radiance * (S2_PI * R * R / lp.pdf);
                    ok = R > 0.f;
                }
                ok = ok && !any_nan(thr) && any_pos(thr);
            }
        }
        const uint32_t q = warp_append(&P.counters[C_QUEUE0], ok);
        if (ok) {
            const PathQueue& Q = P.q[0];
            Q.s0[q] = make_float4(org.x, org.y, org.z, 0.f);
            Q.s1[q] = make_float4(dir.x, dir.y, dir.z, thr.x);
            Q.s2[q] = make_float4(thr.y, thr.z, 0.f, __uint_as_float(0u));
            Q.s3[q] = make_uint4(rng.px, rng.py, rng.seed, rng.ctr);
        }
    }
}

// One light-subpath vertex: camera connection, then continuation (TraceRay / ConnectToCamera /
// sampleDirection<true> of the light pass).
template <bool LAMBERT>
__global__ void __launch_bounds__(128) k_light_shade(PTParams P, uint32_t parity) {
    const uint32_t count = P.counters[parity];
    const PathQueue qi = P.q[parity];
    const PathQueue qo = P.q[1 - parity];
    const DevScene& s = P.scene;
    const bool sn = !(P.flags & S2F_NO_SN);
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t rounded = (count + 31u) & ~31u;
    const float* ci = P.cam_inv;
    const float3 cam = f3(P.cam[3], P.cam[7], P.cam[11]);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rounded; i += stride) {
        bool alive = false, shadow = false;
        float4 n0, n1, n2;
        uint4 n3;
        float3 so_o = f3(0.f), so_d = f3(0.f), so_c = f3(0.f);
        float so_t = 0.f;
        uint32_t so_pix = 0;
        if (i < count) {
            const float4 a = qi.s0[i], b = qi.s1[i], c = qi.s2[i];
            const uint4 rs = qi.s3[i];
            const float4 h = P.hits[i];
            const float3 dir = f3(b.x, b.y, b.z);
            float3 thr = f3(b.w, c.x, c.y);
            const uint32_t meta = __float_as_uint(c.w);
            const uint32_t len = (meta & 0xffu) + 1u;
            Rng rng;
            rng.px = rs.x; rng.py = rs.y; rng.seed = rs.z; rng.ctr = rs.w; rng.pcg32 = (P.flags & S2F_PCG32) != 0;
            const uint32_t tri = __float_as_uint(h.y);
            if (tri != 0xffffffffu && len < P.max_len) {
                const float4 ra = __ldg(s.tris + 3 * (size_t)tri), rb = __ldg(s.tris + 3 * (size_t)tri + 1);
                const uint32_t inst = __float_as_uint(ra.w), prim = __float_as_uint(rb.w);
                SD sd = make_shading(s, inst, prim, h.z, h.w, sn);
                if (!(P.flags & S2F_NO_NORMAL_MAPS)) apply_normal_map(s, sd);
                const Mat m = load_material(s, sd.mat, sd.uv);
                const float3 in = sd.to_local(-dir);
                if (any_pos(m.base())) {
                    const bool sing = mat_singular<LAMBERT>(m);
                    if (!sing && len + 1 >= P.min_len) {
                        // ConnectToCamera: project, evaluate the BSDF toward the camera and convert the
                        // camera's image-plane pdf to this vertex's area measure
                        const float3 pw = sd.pos;
                        const float3 pc = f3(ci[0] * pw.x + ci[1] * pw.y + ci[2] * pw.z + ci[3],
                                             ci[4] * pw.x + ci[5] * pw.y + ci[6] * pw.z + ci[7],
                                             ci[8] * pw.x + ci[9] * pw.y + ci[10] * pw.z + ci[11]);
                        float2 raster;
                        if (camera_to_raster(P.proj, P.imin, P.imax, pc, raster)) {
                            const float cos_cam = fabsf(pc.z) / length(pc);
                            float3 to_cam = cam - pw;
                            const float dist = length(to_cam);
                            to_cam = to_cam / dist;
                            const float3 out = sd.to_local(to_cam);
                            const float cos_out = fabsf(out.z);
                            float3 f; float fwd, rev;
                            bsdf_eval<LAMBERT>(m, in, out, f, fwd, rev);
                            f = f * snc_adjoint(sd, in, out);
                            const float ipd = P.lt_image_plane_dist / cos_cam;
                            const float image_to_surface = (ipd * ipd / cos_cam) * cos_out / (dist * dist);
                            // thr f / (subpaths * surfaceToImageFactor * cos_out)
                            const float k = image_to_surface / ((float)P.lt_paths * cos_out);
                            const float3 contrib = thr * f * k;
                            const int px = (int)floorf(raster.x) - P.imin[0], py = (int)floorf(raster.y) - P.imin[1];
                            if (any_pos(contrib) && !any_nan(contrib) && px >= 0 && py >= 0 && px < (int)P.width &&
                                py < (int)P.height) {
                                shadow = true;
                                so_o = ray_offset(pw, sd.gn, to_cam);
                                so_d = to_cam;
                                so_t = dist;
                                so_c = contrib;
                                so_pix = (uint32_t)py * P.width + (uint32_t)px;
                            }
                        }
                    }
                    // continuation: Russian roulette, then BSDF sampling with the adjoint correction
                    const float cp = (P.flags & S2F_NO_RR) ? 1.f : fminf(1.f, cont_prob(m));
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
                        fwd *= cp;
                        thr = thr * refl / fwd;
                        thr = thr * snc_adjoint(sd, in, sdir);
                        const float3 wd = sd.to_world(sdir);
                        const float3 nd = unpack_normal(pack_normal(wd));
                        const float3 org = ray_offset(sd.pos, sd.gn, wd);
                        if (any_nan(thr)) {
                            atomicAdd(&P.stats[S_NAN], 1ull);
                        } else if (any_pos(thr)) {
                            alive = true;
                            n0 = make_float4(org.x, org.y, org.z, 0.f);
                            n1 = make_float4(nd.x, nd.y, nd.z, thr.x);
                            n2 = make_float4(thr.y, thr.z, 0.f, __uint_as_float((meta & ~0xffu) | len));
                            n3 = make_uint4(rng.px, rng.py, rng.seed, rng.ctr);
                        }
                    }
                }
            }
        }
        const uint32_t qo_i = warp_append(&P.counters[1 - parity], alive);
        if (alive) { qo.s0[qo_i] = n0; qo.s1[qo_i] = n1; qo.s2[qo_i] = n2; qo.s3[qo_i] = n3; }
        const uint32_t si = warp_append(&P.counters[sh_counter(P)], shadow);
        if (shadow) {
            P.sh_o[si] = make_float4(so_o.x, so_o.y, so_o.z, so_t);
            P.sh_d[si] = make_float4(so_d.x, so_d.y, so_d.z, __uint_as_float(so_pix));
            P.sh_c[si] = make_float4(so_c.x, so_c.y, so_c.z, 0.f);
        }
    }
}

}  // namespace s2
