// Differentiable rendering by adjoint path replay (no counterpart in the reference): the same
// unidirectional path tracer with NEE + MIS as the wavefront renderer (same random-number stream,
// path-length gates, MIS and Russian roulette), in wavefront form over the renderer's own queues
// and closest-hit kernel (one thread per queued path in the shading step), with textured
// material parameters kept in f32 (no 8-bit requantisation, so the image is differentiable in the
// texels).  The adjoint replays every path from its seed twice (Vicini et al. 2021, path replay
// backpropagation): the first replay gives the path's radiance L, the second walks the path again
// and, at every vertex, turns the image adjoint dL/dI into texel gradients:
//   * NEE at vertex j:        dI += T_j Le w / p * df_j(w_light)   and, for the environment,
//                             dI += T_j f_j w / p * dLe;
//   * continuation at j:      dI += (L - L_<=j) / f_j(w_sampled) * df_j(w_sampled)
//                             (every later contribution carries the factor f_j / p_j);
//   * environment hits:       dI += T w * dLe.
// Sampling densities, MIS weights and Russian-roulette probabilities are held constant ("detached"),
// which keeps each term an unbiased estimate of the derivative of the pixel integral.  BSDF partials
// are analytic for the Lambertian model and central differences (f32, step 1e-3) for Disney.
#pragma once
#include "s2_shade_kernel.cuh"

namespace s2 {

// Material with f32 parameters: the record's 8-bit values modulated by the textures in f32.
struct MatF {
    float3 b, e;
    float spec, shn, metal, rough, aniso, subs, cc, ccg, trans, eta;
    S2D float3 base() const { return b; }
    S2D float3 emission() const { return e; }
    S2D float specular() const { return spec; }
    S2D float sheen() const { return shn; }
    S2D float metallic() const { return metal; }
    S2D float roughness() const { return rough; }
    S2D float anisotropic() const { return aniso; }
    S2D float subsurface() const { return subs; }
    S2D float clearcoat() const { return cc; }
    S2D float clearcoat_gloss() const { return ccg; }
    S2D float transmission() const { return trans; }
    S2D float eta1() const { return eta; }
};

// The four texels of a bilinear lookup (same footprint and weights as sample_image).
struct Taps {
    uint32_t img;       // 0xffffffff: no texture
    uint32_t idx[4];
    float w[4];
};

S2D void bilinear_taps(const DevImage& im, uint32_t img, float2 uv, Taps& t) {
    const float x = uv.x * im.width - 0.5f, y = uv.y * im.height - 0.5f;
    const float fx = floorf(x), fy = floorf(y);
    const float ax = x - fx, ay = y - fy;
    int x0 = (int)fx, y0 = (int)fy;
    const int W = (int)im.width, H = (int)im.height;
    x0 %= W; if (x0 < 0) x0 += W;
    y0 %= H; if (y0 < 0) y0 += H;
    const int x1 = (x0 + 1) % W, y1 = (y0 + 1) % H;
    t.img = img;
    t.idx[0] = (uint32_t)(y0 * W + x0); t.idx[1] = (uint32_t)(y0 * W + x1);
    t.idx[2] = (uint32_t)(y1 * W + x0); t.idx[3] = (uint32_t)(y1 * W + x1);
    t.w[0] = (1 - ax) * (1 - ay); t.w[1] = ax * (1 - ay); t.w[2] = (1 - ax) * ay; t.w[3] = ax * ay;
}

// LoadMaterial (material.hlsli:15-46) in f32.  tb / tr: the base-colour and packed[2] (metallic,
// roughness, anisotropic, subsurface) texture taps; base_rec / rough_rec: the record's values.
S2D MatF load_material_f(const DevScene& s, uint32_t addr, float2 uv, Taps& tb, Taps& tr, float3& base_rec,
                         float& rough_rec) {
    const uint4 a = *(const uint4*)(s.material_data + addr);
    const uint4 img = *(const uint4*)(s.material_data + addr + 16);
    MatF m;
    m.b = f3(un8(a.x, 0), un8(a.x, 8), un8(a.x, 16));
    m.spec = un8(a.x, 24);
    m.e = f3(un8(a.y, 0), un8(a.y, 8), un8(a.y, 16)) * ld_f32(s.material_data, addr + 32);
    m.shn = un8(a.y, 24);
    m.metal = un8(a.z, 0); m.rough = un8(a.z, 8); m.aniso = un8(a.z, 16); m.subs = un8(a.z, 24);
    m.cc = un8(a.w, 0); m.ccg = un8(a.w, 8); m.trans = un8(a.w, 16);
    float eta8 = un8(a.w, 24);
    base_rec = m.b;
    rough_rec = m.rough;
    tb.img = tr.img = 0xffffffffu;
    const uint32_t n = s.image_count;
    if (img.x < n) {
        bilinear_taps(s.images[img.x], img.x, uv, tb);
        const float4 t = sample_image(s.images[img.x], uv);
        m.b = m.b * f3(t.x, t.y, t.z);
    }
    if (img.y < n) {
        const float4 t = sample_image(s.images[img.y], uv);
        m.e = m.e * f3(t.x, t.y, t.z);
    }
    if (img.z < n) {
        bilinear_taps(s.images[img.z], img.z, uv, tr);
        const float4 t = sample_image(s.images[img.z], uv);
        m.metal *= t.x;
        m.rough = 1.f - (1.f - m.rough) * (1.f - t.y);  // roughness modulated as smoothness
        m.aniso *= t.z;
        m.subs *= t.w;
    }
    if (img.w < n) {
        const float4 t = sample_image(s.images[img.w], uv);
        m.cc *= t.x; m.ccg *= t.y; m.trans *= t.z; eta8 *= t.w;
    }
    m.eta = eta8 + 1.f;
    return m;
}

struct DiffArgs {
    DevScene scene;
    float proj[8];
    int imin[2], imax[2];
    float cam[12];
    uint32_t width, height, pixels, spp;
    uint32_t min_len, max_len, flags, frame_seed;
    float out_scale;                  // 2^exposure / spp
    float4* image;                    // forward: mean radiance * 2^exposure per pixel
    float4* path_l;                   // forward: radiance of every path, [pixel][sample]
    const float4* d_image;            // adjoint: dLoss / d image
    float4* grad;                     // adjoint: texel gradients of every image, concatenated
    const uint32_t* grad_offset;      // first texel of image k in `grad`
    unsigned long long* rays;         // [0] extension rays, [1] shadow rays
    int* status;                      // bit 0: traversal stack overflow
};

S2D void add_grad(const DiffArgs& A, const Taps& t, float3 g) {
    if (t.img == 0xffffffffu) return;
    float4* base = A.grad + A.grad_offset[t.img];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float* p = (float*)(base + t.idx[k]);
        if (g.x != 0.f) atomicAdd(p + 0, t.w[k] * g.x);
        if (g.y != 0.f) atomicAdd(p + 1, t.w[k] * g.y);
        if (g.z != 0.f) atomicAdd(p + 2, t.w[k] * g.z);
    }
}
S2D void add_grad_y(const DiffArgs& A, const Taps& t, float g) {
    if (t.img == 0xffffffffu || g == 0.f) return;
    float4* base = A.grad + A.grad_offset[t.img];
#pragma unroll
    for (int k = 0; k < 4; ++k) atomicAdd((float*)(base + t.idx[k]) + 1, t.w[k] * g);
}

// Environment texel gradients for radiance weight `g` (dLoss/dLe per channel) in direction `dir`.
S2D void env_grad(const DiffArgs& A, float3 dir, float3 g) {
    const DevScene& s = A.scene;
    if (!has_env(s)) return;
    const float4 rec = *(const float4*)(s.material_data + s.env_address);
    const uint32_t img = __float_as_uint(rec.w);
    if (img >= s.image_count) return;
    Taps t;
    bilinear_taps(s.images[img], img, cartesian_to_spherical_uv(dir), t);
    add_grad(A, t, f3(rec.x * g.x, rec.y * g.y, rec.z * g.z));
}

// dLoss / d(base colour) and d(roughness) of the BSDF value at (in, out) weighted per channel by y,
// pushed to the texels of the vertex's textures.
template <bool LAMBERT>
S2D void material_grads(const DiffArgs& A, const MatF& m, float3 in, float3 out, float3 y, const Taps& tb, const Taps& tr,
                        float3 base_rec, float rough_rec) {
    if (tb.img != 0xffffffffu) {
        float3 g;
        if (LAMBERT) {
            const float c = (in.z * out.z < 0.f) ? 0.f : fabsf(out.z) / S2_PI;
            g = y * c;
        } else {
            const float h = 1e-3f;
            float gg[3];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                MatF mp = m, mm = m;
                float* bp = &mp.b.x;
                float* bm = &mm.b.x;
                bp[j] += h; bm[j] -= h;
                const float3 fp = disney_eval(mp, in, out), fm = disney_eval(mm, in, out);
                gg[j] = dot(y, (fp - fm) / (2.f * h));
            }
            g = f3(gg[0], gg[1], gg[2]);
        }
        add_grad(A, tb, f3(g.x * base_rec.x, g.y * base_rec.y, g.z * base_rec.z));
    }
    if (!LAMBERT && tr.img != 0xffffffffu && rough_rec < 1.f) {
        const float h = 1e-3f;
        const float lo = fmaxf(m.rough - h, 0.f), hi = fminf(m.rough + h, 1.f);
        if (hi > lo) {
            MatF mp = m, mm = m;
            mp.rough = hi; mm.rough = lo;
            const float3 df = (disney_eval(mp, in, out) - disney_eval(mm, in, out)) / (hi - lo);
            add_grad_y(A, tr, dot(y, df) * (1.f - rough_rec));
        }
    }
}

// Wavefront state beside the renderer's queues (PTParams.q): the adjoint replay's running radiance
// (moved with its path, by queue parity), the NEE visibility the first replay found, and the
// gradient records the adjoint replay appends for k_diff_grads.
struct DiffQueues {
    float4* L[2];           // adjoint replay: radiance gathered so far, by queue parity
    uint32_t* vis;          // bit (len - 1) & 31 of word (len - 1) >> 5 of path p: vis[word * paths + p]
    uint32_t paths;         // pixels x spp
    float4* grec;           // gradient records, 3 float4 each (see push_grad)
    uint32_t* gcount;       // records appended this bounce
};

// Slot in a queue for the calling lane, one atomic per group of converged lanes (opportunistic
// warp aggregation; valid in divergent code).
S2D uint32_t append_active(uint32_t* counter) {
    const uint32_t mask = __activemask();
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}

// Gradient record: {in.xyz, uv.x}, {out.xyz, uv.y}, {y.xyz, material address} for the BSDF value at
// (in, out) of the material at uv weighted by y; material address 0xffffffff: environment texels in
// direction in, weighted by y.
S2D void push_grad(const DiffQueues& Q, uint32_t mat, float2 uv, float3 in, float3 out, float3 y) {
    const uint32_t k = append_active(Q.gcount);
    float4* r = Q.grec + 3 * (size_t)k;
    r[0] = make_float4(in.x, in.y, in.z, uv.x);
    r[1] = make_float4(out.x, out.y, out.z, uv.y);
    r[2] = make_float4(y.x, y.y, y.z, __uint_as_float(mat));
}
S2D void push_env_grad(const DiffQueues& Q, float3 dir, float3 y) {
    push_grad(Q, 0xffffffffu, make_float2(0.f, 0.f), dir, f3(0.f), y);
}

S2D float3 add_rn(float3 a, float3 b) { return f3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)); }

// The work at one path vertex, after the closest-hit query of the ray (org, dir): increments len,
// adds the vertex's emission to L, makes the NEE estimate and samples the continuation (org, dir,
// thr, dir_pdf updated; returns false when the path ends).  adj = false (the forward): the NEE
// shadow ray goes to the renderer's shadow queue, whose k_diff_occlude adds its contribution to
// the path's radiance and records the visibility.  adj = true (the adjoint replay): the visibility
// comes from the forward's record, the contribution is added to L here, and the vertex's gradient
// terms for the image adjoint `delta` (ltot: the path's radiance from the forward) go to the
// gradient queue.  Not inlined, and the adjoint is a run-time argument, so both replays run the
// same machine code and take the same decisions.
template <bool LAMBERT>
__device__ __noinline__ bool diff_vertex(const DiffArgs& A, const PTParams& P, const DiffQueues& Q, const TravHit& h,
                                         uint32_t path, uint32_t& len, float3& org, float3& dir, float3& thr, float3& L,
                                         float& dir_pdf, Rng& rng, bool adj, float3 ltot, float3 delta, uint32_t& shadow_rays) {
    const DevScene& s = A.scene;
    const bool nee = !(A.flags & S2F_NO_NEE), sn = !(A.flags & S2F_NO_SN);
    len++;
    if (h.tri == 0xffffffffu) {
        // environment (TraceRay, testrenderer.slang:1036-1054)
        float env_pdf = 0.f;
        const float3 le = eval_env(s, dir, env_pdf);
        const float3 e = len >= A.min_len ? thr * le : f3(0.f);
        if (any_pos(e)) {
            float w = 1.f;
            if (len > 1 && nee && dir_pdf > 0.f) {
                const float lp = (A.flags & S2F_REF_ENV_MIS) ? (S2_INV_PI / pow2(s.scene_sphere.w)) : env_pdf;
                w = mis_w(dir_pdf, lp);
            }
            if (w > 0.f) {
                L = add_rn(L, e * w);
                if (adj) push_env_grad(Q, dir, delta * thr * w);
            }
        }
        return false;
    }
    SD sd = make_shading(s, h.instance, h.primitive, h.b1, h.b2, sn);
    if (!(A.flags & S2F_NO_NORMAL_MAPS)) apply_normal_map(s, sd);
    const float isect_dist = half_round(h.t);
    const float isect_pdfa = half_round(light_pdfa(s, h.instance, sd.area));
    Taps tb, tr;
    float3 base_rec;
    float rough_rec;
    const MatF m = load_material_f(s, sd.mat, sd.uv, tb, tr, base_rec, rough_rec);
    const bool textured = tb.img != 0xffffffffu || tr.img != 0xffffffffu;  // else no texel has a gradient
    const float3 in = sd.to_local(-dir);
    const float cos_in = fabsf(in.z);
    if (in.z > 0.f) {
        const float3 e = thr * m.emission();
        if (any_pos(e) && len >= A.min_len) {
            float w = 1.f;
            if (len > 1 && nee && dir_pdf > 0.f) w = mis_w(dir_pdf * (cos_in / pow2(isect_dist)), isect_pdfa);
            if (w > 0.f) L = add_rn(L, e * w);
        }
    }
    if (!(len < A.max_len && any_pos(m.base()))) return false;
    const bool sing = mat_singular<LAMBERT>(m);
    const float cp = (A.flags & S2F_NO_RR) ? 1.f : cont_prob(m);
    // NEE (ConnectToLight, testrenderer.slang:751-779), same stream use as the wavefront shade
    if (!sing && nee) {
        if (len + 1 < A.min_len) {
            rng.skip();
        } else {
            const float4 x = rng.next_float();
            const Illum r = sample_illum(s, x, sd.pos, sn);
            if (!(all_nonpos(r.radiance) || r.pdf <= 0.f)) {
                const float AtoW = r.finite ? pow2(r.dist) / r.cos_light : 1.f;
                const float dpw = r.pdf * AtoW;
                const float3 out = sd.to_local(r.dir);
                float3 f; float fwd, rev;
                bsdf_eval<LAMBERT>(m, in, out, f, fwd, rev);
                f = f * sd.snc(in, out);
                fwd *= cp;
                const float3 contrib = thr * r.radiance * f / dpw;
                const float w = mis_w(r.pdf, fwd / AtoW);
                if (w > 0.f && !all_nonpos(contrib)) {
                    const float3 c = f3(fmaxf(contrib.x * w, 0.f), fmaxf(contrib.y * w, 0.f), fmaxf(contrib.z * w, 0.f));
                    if (!adj) {
                        const float3 o = ray_offset(sd.pos, sd.gn, r.dir);
                        const uint32_t q = append_active(&P.counters[C_SHADOW]);
                        P.sh_o[q] = make_float4(o.x, o.y, o.z, adjust_distance(r.dist));
                        P.sh_d[q] = make_float4(r.dir.x, r.dir.y, r.dir.z, __uint_as_float(path));
                        P.sh_c[q] = make_float4(c.x, c.y, c.z, __uint_as_float(len));
                        shadow_rays++;
                    } else if (Q.vis[(size_t)((len - 1) >> 5) * Q.paths + path] & (1u << ((len - 1) & 31u))) {
                        L = add_rn(L, c);
                        const float k = w / dpw;
                        if (textured) push_grad(Q, sd.mat, sd.uv, in, out, delta * thr * r.radiance * k);
                        if (!r.finite) push_env_grad(Q, r.dir, delta * thr * f * k);
                    }
                }
            }
        }
    }
    if (!(A.flags & S2F_NO_RR)) {
        const float4 u = rng.next_float();
        if (u.x > fminf(1.f, cp)) return false;
    }
    const float4 rnd = rng.next_float();
    float3 sdir, refl;
    float fwd, rev, rough;
    bsdf_sample<LAMBERT>(m, in, rnd, sdir, refl, fwd, rev, rough);
    if (adj) {
        // every later contribution carries refl / fwd: d/dtheta = (L - L_so_far) * d refl / refl
        const float3 after = ltot - L;
        const float3 y = f3(refl.x > 0.f ? delta.x * after.x / refl.x : 0.f, refl.y > 0.f ? delta.y * after.y / refl.y : 0.f,
                            refl.z > 0.f ? delta.z * after.z / refl.z : 0.f);
        if (textured && any_pos(f3(fabsf(y.x), fabsf(y.y), fabsf(y.z))))
            push_grad(Q, sd.mat, sd.uv, in, sdir, y);
    }
    const float cpm = (A.flags & S2F_NO_RR) ? 1.f : cp;
    fwd *= cpm;
    thr = thr * refl / fwd;
    dir_pdf = (rough == 0.f || sing) ? 0.f : half_round(fwd);
    thr = thr * sd.snc(in, sdir);
    const float3 wd = sd.to_world(sdir);
    org = ray_offset(sd.pos, sd.gn, wd);
    dir = unpack_normal(pack_normal(wd));
    return !(any_nan(thr) || !any_pos(thr));
}

S2D void diff_count(const DiffArgs& A, uint32_t ext, uint32_t shd, bool overflow) {
    // warp sums of the ray counts, one 64-bit atomic pair per warp
    for (int o = 16; o > 0; o >>= 1) { ext += __shfl_xor_sync(0xffffffffu, ext, o); shd += __shfl_xor_sync(0xffffffffu, shd, o); }
    if ((threadIdx.x & 31u) == 0) { atomicAdd(A.rays, (unsigned long long)ext); atomicAdd(A.rays + 1, (unsigned long long)shd); }
    if (overflow) atomicOr(A.status, 1);
}

// Camera paths base .. base + n - 1 into queue 0.  Path ids run over pixels (row-major), then
// samples (path = pixel x spp + sample), so a warp takes the samples of one or a few neighbouring
// pixels, their camera rays traverse together and a pixel's radiances are contiguous in path_l.
// The forward zeroes each path's radiance in path_l and its visibility words; the adjoint skips
// paths of pixels whose adjoint is zero, as their replay adds nothing.
__global__ void k_diff_gen(const __grid_constant__ DiffArgs A, PTParams P, DiffQueues Q, uint32_t base, uint32_t n, int adj) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool want = false;
    uint32_t path = 0, px = 0, py = 0, k = 0;
    if (i < n) {
        path = base + i;
        const uint32_t pix = path / A.spp;
        k = path - pix * A.spp;
        px = pix % A.width; py = pix / A.width;
        want = true;
        if (adj) {
            const float4 d = A.d_image[pix];
            want = d.x != 0.f || d.y != 0.f || d.z != 0.f;
        } else {
            A.path_l[path] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (Q.vis)
                for (uint32_t w = 0; w < (A.max_len + 31u) >> 5; ++w) Q.vis[(size_t)w * Q.paths + path] = 0u;
        }
    }
    const uint32_t q = warp_append(&P.counters[C_QUEUE0], want);
    if (!want) return;
    Rng rng = make_rng(px, py, A.frame_seed + k, (A.flags & S2F_PCG32) != 0);
    float ox = 0.5f, oy = 0.5f;
    if (A.flags & S2F_JITTER) { const float4 f = rng.next_float(); ox = f.x; oy = f.y; }
    const float3 dir = camera_dir(A.proj, A.imin, A.imax, A.cam, px, py, ox, oy);
    const PathQueue& Qo = P.q[0];
    Qo.s0[q] = make_float4(A.cam[3], A.cam[7], A.cam[11], 0.f);
    Qo.s1[q] = make_float4(dir.x, dir.y, dir.z, 1.f);
    Qo.s2[q] = make_float4(1.f, 1.f, __uint_as_float(path), __uint_as_float(0u));
    Qo.s3[q] = make_uint4(rng.px, rng.py, rng.seed, rng.ctr);
    if (adj) Q.L[0][q] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Counters before a bounce: the queue about to be traced counts as extension rays; the other
// queue, the shadow queue, the gradient records and the traversal work counters restart.
__global__ void k_diff_bounce(const __grid_constant__ DiffArgs A, PTParams P, DiffQueues Q, uint32_t parity) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    atomicAdd(A.rays, (unsigned long long)P.counters[parity]);
    P.counters[1 - parity] = 0;
    P.counters[C_SHADOW] = 0;
    P.counters[C_WORK_EXT] = 0;
    P.counters[C_WORK_OCC] = 0;
    *Q.gcount = 0;
}

template <bool LAMBERT>
__global__ void __launch_bounds__(128, 8) k_diff_shade(const __grid_constant__ DiffArgs A, const __grid_constant__ PTParams P,
                                                    DiffQueues Q, uint32_t parity, int adj) {
    const uint32_t count = P.counters[parity];
    const PathQueue qi = P.q[parity], qo = P.q[1 - parity];
    const uint32_t rounded = (count + 31u) & ~31u;
    uint32_t shd = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rounded; i += gridDim.x * blockDim.x) {
        bool alive = false;
        float4 n0, n1, n2, nl;
        uint4 n3;
        if (i < count) {
            const float4 a = qi.s0[i], b = qi.s1[i], c = qi.s2[i];
            const uint4 rs = qi.s3[i];
            const float4 hv = P.hits[i];
            const uint32_t path = __float_as_uint(c.z);
            const float4 l4 = adj ? Q.L[parity][i] : A.path_l[path];
            float3 org = f3(a.x, a.y, a.z), dir = f3(b.x, b.y, b.z), thr = f3(b.w, c.x, c.y), L = f3(l4.x, l4.y, l4.z);
            float dir_pdf = a.w;
            uint32_t len = __float_as_uint(c.w);
            Rng rng;
            rng.px = rs.x; rng.py = rs.y; rng.seed = rs.z; rng.ctr = rs.w; rng.pcg32 = (A.flags & S2F_PCG32) != 0;
            TravHit h;
            h.t = hv.x;
            h.tri = __float_as_uint(hv.y);
            h.b1 = hv.z; h.b2 = hv.w;
            h.instance = h.primitive = 0xffffffffu;
            if (h.tri != 0xffffffffu) {
                const float4 t0 = P.scene.tris[3 * (size_t)h.tri], t1 = P.scene.tris[3 * (size_t)h.tri + 1];
                h.instance = __float_as_uint(t0.w);
                h.primitive = __float_as_uint(t1.w);
            }
            float3 ltot = f3(0.f), delta = f3(0.f);
            if (adj) {
                const uint32_t pix = path / A.spp;
                const float4 lt = A.path_l[path], d = A.d_image[pix];
                ltot = f3(lt.x, lt.y, lt.z);
                delta = f3(d.x, d.y, d.z) * A.out_scale;
            }
            alive = diff_vertex<LAMBERT>(A, P, Q, h, path, len, org, dir, thr, L, dir_pdf, rng, adj != 0, ltot, delta, shd);
            if (!adj) A.path_l[path] = make_float4(L.x, L.y, L.z, 0.f);
            if (alive) {
                n0 = make_float4(org.x, org.y, org.z, dir_pdf);
                n1 = make_float4(dir.x, dir.y, dir.z, thr.x);
                n2 = make_float4(thr.y, thr.z, __uint_as_float(path), __uint_as_float(len));
                n3 = make_uint4(rng.px, rng.py, rng.seed, rng.ctr);
                nl = make_float4(L.x, L.y, L.z, 0.f);
            }
        }
        const uint32_t o = warp_append(&P.counters[1 - parity], alive);
        if (alive) {
            qo.s0[o] = n0; qo.s1[o] = n1; qo.s2[o] = n2; qo.s3[o] = n3;
            if (adj) Q.L[1 - parity][o] = nl;
        }
    }
    diff_count(A, 0u, shd, false);
}

// The forward's shadow rays, on the renderer's persistent any-hit loop: an unoccluded ray adds its
// contribution to its path's radiance (one shadow ray per path and bounce, so no other thread
// touches the path meanwhile) and, for the adjoint, sets its visibility bit.
__global__ void __launch_bounds__(kTravBlock) k_diff_occlude(const __grid_constant__ DiffArgs A, const __grid_constant__ PTParams P,
                                                            DiffQueues Q) {
    __shared__ uint2 stack[S2_STACK_SMEM * kTravBlock];
    occlude_queue<false>(P, C_SHADOW, stack, [&](uint32_t ray) {
        const float4 cc = P.sh_c[ray];
        const uint32_t path = __float_as_uint(P.sh_d[ray].w);
        const float4 l = A.path_l[path];
        A.path_l[path] = make_float4(__fadd_rn(l.x, cc.x), __fadd_rn(l.y, cc.y), __fadd_rn(l.z, cc.z), 0.f);
        if (Q.vis) {
            const uint32_t j = __float_as_uint(cc.w) - 1u;
            Q.vis[(size_t)(j >> 5) * Q.paths + path] |= 1u << (j & 31u);
        }
    });
}

// The adjoint replay's gradient records of one bounce: the BSDF partials of the record's material
// (reloaded from its address and uv) pushed to the texels, or the environment texels' gradient.
template <bool LAMBERT>
__global__ void __launch_bounds__(128) k_diff_grads(const __grid_constant__ DiffArgs A, DiffQueues Q) {
    const uint32_t count = *Q.gcount;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float4* r = Q.grec + 3 * (size_t)i;
        const float4 r0 = r[0], r1 = r[1], r2 = r[2];
        const uint32_t mat = __float_as_uint(r2.w);
        const float3 y = f3(r2.x, r2.y, r2.z);
        if (mat == 0xffffffffu) {
            env_grad(A, f3(r0.x, r0.y, r0.z), y);
            continue;
        }
        Taps tb, tr;
        float3 base_rec;
        float rough_rec;
        const MatF m = load_material_f(A.scene, mat, make_float2(r0.w, r1.w), tb, tr, base_rec, rough_rec);
        material_grads<LAMBERT>(A, m, f3(r0.x, r0.y, r0.z), f3(r1.x, r1.y, r1.z), y, tb, tr, base_rec, rough_rec);
    }
}

// image[pixel] = sum of the pixel's path radiances in sample order * 2^exposure / spp.
__global__ void k_diff_resolve(const __grid_constant__ DiffArgs A) {
    const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= A.pixels) return;
    float3 sum = f3(0.f);
    for (uint32_t k = 0; k < A.spp; ++k) {
        const float4 l = A.path_l[(size_t)pix * A.spp + k];
        sum = sum + f3(l.x, l.y, l.z);
    }
    A.image[pix] = make_float4(sum.x * A.out_scale, sum.y * A.out_scale, sum.z * A.out_scale, 1.f);
}

}  // namespace s2
