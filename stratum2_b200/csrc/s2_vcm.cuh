// Vertex connection and merging (the reference's VCM renderer, vcm.slang:1-1238, itself after
// SmallVCM's vertexcm.hxx; MIS quantities dVCM / dVC / dVM of Georgiev et al. 2012, "Light
// transport simulation with vertex connection and merging", tech. rep. eqs. 31-55).  One thread per
// light subpath, then one per camera path, both on the shared BVH8 traversal:
//   * light pass (GenerateLightPaths, vcm.slang:1145-1219): emission sample, random walk with the
//     adjoint BSDF, every non-singular vertex stored (80-byte LightVertex) and connected to the camera;
//   * grid build: the stored vertices sorted by the hash of their merge cell (cells 2r wide, so a
//     query visits the 2x2x2 cells around it);
//   * camera pass (GenerateCameraPaths, vcm.slang:880-1009): per vertex the emission hit, direct
//     illumination, connections to the vertices of light subpath (pixel mod n_light) or to one random
//     cached vertex (LVC), and merging with the light vertices within the merge radius.
// All contributions land in 64-bit fixed-point pixel totals, so images do not depend on the order of
// the atomic additions.  The environment is black and never sampled (the reference's
// GetBackgroundRadiance returns zero radiance, vcm.hlsli:303-313), so the host hands these kernels a
// scene without one.
#pragma once
#include "s2_light_trace.cuh"

namespace s2 {

// VcmAlgorithmType (compat/vcm.h:103-132)
enum : uint32_t { VCM_PT = 0, VCM_LT = 1, VCM_PPM = 2, VCM_BPM = 3, VCM_BPT = 4, VCM_VCM = 5 };

// One stored light-subpath vertex (PackedVcmVertex, compat/vcm.h:75-85, with the hit kept as
// barycentrics so make_shading rebuilds the same shading frame): 80 bytes.
struct LightVertex {
    float4 a;  // position, continuation probability of its material
    float4 b;  // throughput, dVCM
    float4 c;  // dVC, dVM, packed world direction toward the previous vertex (bits), path length (bits)
    uint4 d;   // instance, primitive, barycentrics b1, b2 (bits)
    float4 e;  // the subpath's area-measure pdf up to this vertex (mPathPdfA), unused x 3
};

// One stored light-vertex-cache reservoir (LVCReservoir, compat/vcm.h:92-101): the selected light
// vertex by value (the cache is rebuilt every iteration), the camera vertex it was resampled at (on
// its triangle, with the MIS quantities its connections use) and the reservoir's M, integration
// weight and target pdf.  128 bytes.  A reservoir without a sample keeps a zero-throughput vertex.
struct LvcRecord {
    LightVertex lv;
    float3 local_pos;     // camera vertex, object space of its instance
    uint32_t instance;
    uint32_t primitive;
    uint32_t in_dir;      // packed world direction toward the previous camera vertex
    uint32_t len;         // camera vertices so far
    float dvcm;
    float dvc;
    float M;
    float W;
    float phat;
};
static_assert(sizeof(LvcRecord) == 128, "LvcRecord is two 64-byte lines");

struct VcmArgs {
    DevScene scene;
    float proj[8];
    int imin[2], imax[2];
    float cam[12], cam_inv[12], prev_inv[12];
    float image_plane_dist;        // ViewData::imagePlaneDist: |image height| / (2 tan(vfov / 2))
    uint32_t width, height, pixels;
    uint32_t n_light;              // light subpaths per iteration (mLightSubPathCount)
    uint32_t min_len, max_len, flags, seed;
    uint32_t use_vc, use_vm, ppm, light_trace_only, path_trace_only, lvc;
    uint32_t debug_paths, debug_unweighted, debug_cam, debug_light;
    float merge_radius, vm_weight, vc_weight, vm_norm, cell_size;
    LightVertex* lv;               // slot k * n_light + p: vertex k of light subpath p
    uint32_t* lv_count;            // stored vertices per light subpath
    uint32_t lv_slots;             // n_light * (max_len - 1)
    // merge grid: vertex slots sorted by cell hash, [start, end) per hash bucket
    uint32_t* grid_key;
    uint32_t* grid_val;
    const uint32_t* grid_slot;
    uint32_t* grid_start;
    uint32_t* grid_end;
    uint32_t grid_mask;
    // light vertex cache: the stored vertices' slots in slot order and their count
    const uint32_t* lvc_list;
    const uint32_t* lvc_total;
    unsigned long long* image_fx;  // 4 x u64 per pixel, 2^-24 fixed point
    float4* aov_albedo;
    uint2* aov_vis;
    float4* aov_depth;
    float2* aov_prev_uv;
    uint2* aov_ids;
    uint32_t write_aovs;
    unsigned long long* counts;    // [0] extension rays, [1] shadow rays, [2] NaN paths
    int* status;                   // bit 0: traversal stack overflow
    // direct-illumination reservoirs (S2_VCM_FLAG_DI_RIS / _DI_REUSE): candidates, M cap, and the
    // world-space grids of this iteration's reservoirs (appended) and the previous one's (read)
    uint32_t di_ris, di_reuse, di_m, di_prev_valid;
    float di_max_m;
    HashGridDev di_cur, di_prev;
    uint32_t lvc_m;                // light-vertex-cache reservoirs (S2_VCM_FLAG_LVC_RIS): candidates, 0 = off
    // their reuse (S2_VCM_FLAG_LVC_REUSE): M cap, this iteration's grid (appended; records in
    // lvc_cur_rec at the grid's data index) and the previous one's (read)
    uint32_t lvc_reuse, lvc_prev_valid;
    float lvc_max_m;
    HashGridDev lvc_cur, lvc_prev;
    LvcRecord* lvc_cur_rec;
    const LvcRecord* lvc_prev_rec;
};

// Mis() (compat/vcm.h:9-11): power heuristic with exponent 2.
S2D float vmis(float x) { return x * x; }

// AddColor / InterlockedAddColor (vcm.hlsli:345-370): the debug filter on (camera, light) vertex
// counts; unweighted debug images replace every MIS weight by 1.
S2D bool vcm_pass(const VcmArgs& A, uint32_t cam_vertices, uint32_t light_vertices) {
    return !A.debug_paths || (cam_vertices == A.debug_cam && light_vertices == A.debug_light);
}
S2D float vcm_w(const VcmArgs& A, float w) { return A.debug_unweighted ? 1.f : w; }

S2D void vcm_splat(const VcmArgs& A, uint32_t pix, float3 v) {
    if (any_nan(v)) { atomicAdd(A.counts + 2, 1ull); return; }
    unsigned long long* t = A.image_fx + 4 * (size_t)pix;
    if (v.x > 0.f) atomicAdd(t + 0, (unsigned long long)__float2ull_rn(v.x * S2_FX_SCALE));
    if (v.y > 0.f) atomicAdd(t + 1, (unsigned long long)__float2ull_rn(v.y * S2_FX_SCALE));
    if (v.z > 0.f) atomicAdd(t + 2, (unsigned long long)__float2ull_rn(v.z * S2_FX_SCALE));
}

struct VcmTrace {
    uint2* stack;
    uint32_t lane_stride;
    uint32_t ext, shadow;
    bool overflow;
    TravCounters ctr;
};

S2D TravHit vcm_closest(const VcmArgs& A, VcmTrace& T, float3 o, float3 d) {
    const SceneAlphaTest alpha{&A.scene, !(A.flags & S2F_NO_ALPHA)};
    TravHit h;
    T.ext++;
    if (!traverse<false, false>(make_trav_ray(o, d, 0.f), S2_INF, A.scene.nodes, A.scene.tris, T.stack, T.lane_stride, h, T.ctr, alpha))
        T.overflow = true;
    return h;
}
S2D bool vcm_visible(const VcmArgs& A, VcmTrace& T, float3 o, float3 d, float tmax) {
    const SceneAlphaTest alpha{&A.scene, !(A.flags & S2F_NO_ALPHA)};
    TravHit h;
    T.shadow++;
    if (!traverse<true, false>(make_trav_ray(o, d, 0.f), tmax, A.scene.nodes, A.scene.tris, T.stack, T.lane_stride, h, T.ctr, alpha))
        T.overflow = true;
    return h.tri == 0xffffffffu;
}

// The subpath state both walks carry (SubPathState, vcm.slang:24-51).
struct SubPath {
    float3 thr;
    float dvcm, dvc, dvm;
    float fwd_pdfw;   // BSDF pdf of the last scattering (infinite after a singular one)
    uint32_t len;
    bool specular;    // every scattering so far was singular
    float pdfa;       // light subpaths: the path's pdf in area measure (mPathPdfA, vcm.slang:114, 1025, 1193)
};

// SampleScattering<Adjoint> (vcm.slang:67-113): Russian roulette, BSDF sampling and the MIS updates
// of tech. rep. eqs. 34-36 (53-55 for a singular sample).  Returns false when the walk ends.
template <bool LAMBERT, bool ADJOINT>
S2D bool vcm_scatter(const VcmArgs& A, const Mat& m, const SD& sd, float3 in, bool sing, Rng& rng, SubPath& p, float3& dir) {
    const float cp = (A.flags & S2F_NO_RR) ? 1.f : cont_prob(m);
    if (!(A.flags & S2F_NO_RR) && rng.next_float().x > cp) return false;
    const float4 rnd = rng.next_float();
    float3 sdir, refl;
    float fwd, rev, rough;
    bsdf_sample<LAMBERT>(m, in, rnd, sdir, refl, fwd, rev, rough);
    refl = refl * (ADJOINT ? snc_adjoint(sd, in, sdir) : sd.snc(in, sdir));
    if (all_nonpos(refl)) return false;
    const float cos_out = fabsf(sdir.z);
    const float dir_pdf = fwd * cp, rev_pdf = rev * cp;
    if (sing || rough == 0.f) {
        p.dvcm = 0.f;
        p.dvc *= vmis(cos_out);
        p.dvm *= vmis(cos_out);
        p.fwd_pdfw = S2_INF;
    } else {
        const float k = vmis(cos_out / dir_pdf);
        p.dvc = k * (p.dvc * vmis(rev_pdf) + p.dvcm + A.vm_weight);
        p.dvm = k * (p.dvm * vmis(rev_pdf) + p.dvcm * A.vc_weight + 1.f);
        p.dvcm = vmis(1.f / dir_pdf);
        p.specular = false;
        p.fwd_pdfw = dir_pdf;
    }
    p.thr = p.thr * refl / dir_pdf;
    p.pdfa *= dir_pdf;
    if (any_nan(p.thr) || !any_pos(p.thr)) return false;
    dir = sd.to_world(sdir);
    return true;
}

// ---------------------------------------------------------------- light pass
// ConnectToCamera (vcm.slang:1040-1110): the light vertex seen through the pinhole, with the
// light-tracing MIS weight of tech. rep. eq. 46.
template <bool LAMBERT>
S2D void vcm_connect_camera(const VcmArgs& A, VcmTrace& T, const Mat& m, const SD& sd, float3 in, const SubPath& p) {
    const float* ci = A.cam_inv;
    const float3 pw = sd.pos;
    const float3 pc = f3(ci[0] * pw.x + ci[1] * pw.y + ci[2] * pw.z + ci[3], ci[4] * pw.x + ci[5] * pw.y + ci[6] * pw.z + ci[7],
                         ci[8] * pw.x + ci[9] * pw.y + ci[10] * pw.z + ci[11]);
    float2 raster;
    if (!camera_to_raster(A.proj, A.imin, A.imax, pc, raster)) return;
    const int px = (int)floorf(raster.x) - A.imin[0], py = (int)floorf(raster.y) - A.imin[1];
    if (px < 0 || py < 0 || px >= (int)A.width || py >= (int)A.height) return;
    if (!vcm_pass(A, 1, p.len + 1)) return;
    const float3 cam = f3(A.cam[3], A.cam[7], A.cam[11]);
    float3 to_cam = cam - pw;
    const float dist = length(to_cam);
    to_cam = to_cam / dist;
    const float3 out = sd.to_local(to_cam);
    float3 f; float fwd, rev;
    bsdf_eval<LAMBERT>(m, in, out, f, fwd, rev);
    f = f * snc_adjoint(sd, in, out);
    if (all_nonpos(f)) return;
    const float cp = (A.flags & S2F_NO_RR) ? 1.f : cont_prob(m);
    const float rev_pdf = rev * cp;
    const float cos_cam = fabsf(pc.z) / length(pc);
    const float ipd = A.image_plane_dist / cos_cam;
    const float image_to_surface = (ipd * ipd / cos_cam) * fabsf(out.z) / (dist * dist);
    const float w_light = vmis(image_to_surface / (float)A.n_light) * (A.vm_weight + p.dvcm + p.dvc * vmis(rev_pdf));
    const float w = A.light_trace_only ? 1.f : vcm_w(A, 1.f / (w_light + 1.f));
    const float3 contrib = p.thr * f * (w * image_to_surface / ((float)A.n_light * fabsf(out.z)));
    if (!any_pos(contrib)) return;
    if (!vcm_visible(A, T, ray_offset(pw, sd.gn, to_cam), to_cam, dist)) return;
    vcm_splat(A, (uint32_t)py * A.width + (uint32_t)px, contrib);
}

template <bool LAMBERT>
__global__ void __launch_bounds__(128) k_vcm_light(const __grid_constant__ VcmArgs A) {
    __shared__ uint2 stack[S2_STACK_SMEM * 128];
    VcmTrace T{stack + threadIdx.x, 128u, 0u, 0u, false, {0, 0}};
    const DevScene& s = A.scene;
    const bool sn = !(A.flags & S2F_NO_SN);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_light; i += gridDim.x * blockDim.x) {
        // VertexCM(index, 16384): light subpath i at pixel index (i mod W, i / W), counter offset 16384
        Rng rng = make_rng(i % A.width, i / A.width, A.seed, (A.flags & S2F_PCG32) != 0);
        if (!rng.pcg32) rng.ctr = 16384u;
        else rng = make_rng(i % A.width, (i / A.width) | 0x80000000u, A.seed, true);
        // GenerateLightSample (vcm.slang:1013-1038)
        const LightPoint lp = sample_light_point(s, rng.next_float(), sn);
        const float4 u = rng.next_float();
        if (!lp.ok || !lp.finite) continue;
        const float3 ld = sample_cos_hemisphere(u.x, u.y);
        const float cos_light = ld.z;
        const float emission_pdfw = lp.pdf * cos_hemisphere_pdfw(cos_light);
        if (!(emission_pdfw > 0.f)) continue;
        float3 t, b;
        make_orthonormal(lp.n, t, b);
        float3 dir = normalize(t * ld.x + b * ld.y + lp.n * ld.z);
        float3 org = ray_offset(lp.pos, lp.n, dir);
        SubPath p;
        p.thr = lp.radiance * (cos_light / emission_pdfw);
        p.dvcm = vmis(lp.pdf / emission_pdfw);
        p.dvc = vmis(cos_light / emission_pdfw);
        p.dvm = p.dvc * A.vc_weight;
        p.fwd_pdfw = 0.f;
        p.len = 1;
        p.specular = true;
        p.pdfa = emission_pdfw;
        uint32_t stored = 0;
        while (true) {
            const TravHit h = vcm_closest(A, T, org, dir);
            if (h.tri == 0xffffffffu) break;
            SD sd = make_shading(s, h.instance, h.primitive, h.b1, h.b2, sn);
            const Mat m = load_material(s, sd.mat, sd.uv);
            if (!any_pos(m.base())) break;  // canEvaluate
            if (!(A.flags & S2F_NO_NORMAL_MAPS)) apply_normal_map(s, sd);
            const float3 in = sd.to_local(-dir);
            // tech. rep. eqs. 31-36, completed at the hit
            const float cos_in = fabsf(in.z);
            p.dvcm *= vmis(h.t * h.t);
            p.dvcm /= vmis(cos_in);
            p.dvc /= vmis(cos_in);
            p.dvm /= vmis(cos_in);
            p.pdfa *= cos_in / (h.t * h.t);
            const bool sing = mat_singular<LAMBERT>(m);
            if (!sing) {
                if ((A.use_vc || A.use_vm) && p.len < A.max_len) {  // StoreLightVertex (vcm.slang:1112-1140)
                    LightVertex v;
                    v.a = make_float4(sd.pos.x, sd.pos.y, sd.pos.z, (A.flags & S2F_NO_RR) ? 1.f : cont_prob(m));
                    v.b = make_float4(p.thr.x, p.thr.y, p.thr.z, p.dvcm);
                    v.c = make_float4(p.dvc, p.dvm, __uint_as_float(pack_normal(-dir)), __uint_as_float(p.len));
                    v.d = make_uint4(h.instance, h.primitive, __float_as_uint(h.b1), __float_as_uint(h.b2));
                    v.e = make_float4(p.pdfa, 0.f, 0.f, 0.f);
                    A.lv[(size_t)stored * A.n_light + i] = v;
                    stored++;
                }
                if ((A.use_vc || A.light_trace_only) && p.len + 1 >= A.min_len && p.len + 1 <= A.max_len)
                    vcm_connect_camera<LAMBERT>(A, T, m, sd, in, p);
            }
            if (p.len + 2 > A.max_len) break;
            if (!vcm_scatter<LAMBERT, true>(A, m, sd, in, sing, rng, p, dir)) break;
            org = ray_offset(sd.pos, sd.gn, dir);
            p.len++;
        }
        if (A.use_vc || A.use_vm) A.lv_count[i] = stored;
    }
    for (int o = 16; o > 0; o >>= 1) { T.ext += __shfl_xor_sync(0xffffffffu, T.ext, o); T.shadow += __shfl_xor_sync(0xffffffffu, T.shadow, o); }
    if ((threadIdx.x & 31u) == 0) { atomicAdd(A.counts, (unsigned long long)T.ext); atomicAdd(A.counts + 1, (unsigned long long)T.shadow); }
    if (T.overflow) atomicOr(A.status, 1);
}

// ---------------------------------------------------------------- merge grid and vertex cache
S2D int3 vcm_cell(const VcmArgs& A, float3 p) {
    return make_int3((int)floorf(p.x / A.cell_size), (int)floorf(p.y / A.cell_size), (int)floorf(p.z / A.cell_size));
}
S2D uint32_t vcm_cell_hash(int3 c) { return pcg_hash((uint32_t)c.x + pcg_hash((uint32_t)c.y + pcg_hash((uint32_t)c.z))); }

// Sort keys of every slot.  Merging: the hash bucket of its vertex's cell, grid_mask + 1 for an
// empty slot.  Light vertex cache: 0 for a stored vertex, 1 for an empty slot (the stable sort then
// lists the cached vertices first, in slot order), with their count in lvc_count.
__global__ void k_vcm_keys(const __grid_constant__ VcmArgs A, unsigned int* lvc_count) {
    const uint32_t rounded = (A.lv_slots + 31u) & ~31u;
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < rounded; slot += gridDim.x * blockDim.x) {
        bool valid = false;
        float3 pos = f3(0.f);
        if (slot < A.lv_slots) {
            const uint32_t k = slot / A.n_light, path = slot - k * A.n_light;
            if (k < A.lv_count[path]) {
                const LightVertex& v = A.lv[slot];
                pos = f3(v.a.x, v.a.y, v.a.z);
                valid = any_pos(f3(v.b.x, v.b.y, v.b.z));
            }
            if (A.lvc) A.grid_key[slot] = valid ? 0u : 1u;
            else A.grid_key[slot] = valid ? (vcm_cell_hash(vcm_cell(A, pos)) & A.grid_mask) : A.grid_mask + 1u;
            A.grid_val[slot] = slot;
        }
        if (A.lvc) {
            const uint32_t ballot = __ballot_sync(0xffffffffu, valid);
            if ((threadIdx.x & 31u) == 0 && ballot) atomicAdd(lvc_count, (unsigned int)__popc(ballot));
        }
    }
}

// [start, end) of every hash bucket in the sorted key array (buckets left empty stay 0, 0).
__global__ void k_vcm_ranges(const __grid_constant__ VcmArgs A, const uint32_t* __restrict__ keys) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < A.lv_slots; i += gridDim.x * blockDim.x) {
        const uint32_t key = keys[i];
        if (key > A.grid_mask) continue;
        if (i == 0 || keys[i - 1] != key) A.grid_start[key] = i;
        if (i + 1 == A.lv_slots || keys[i + 1] != key) A.grid_end[key] = i + 1;
    }
}

// ---------------------------------------------------------------- camera pass
// ConnectVertices (vcm.slang:484-558): camera vertex to light vertex with the MIS weights of tech.
// rep. eqs. 37, 40-41; the visibility ray is traced here unless `vis` is false.
template <bool LAMBERT>
S2D float3 vcm_connect(const VcmArgs& A, VcmTrace& T, const Mat& m, const SD& sd, float3 in, float cp, const SubPath& p,
                       const LightVertex& v, bool vis = true) {
    const DevScene& s = A.scene;
    const bool sn = !(A.flags & S2F_NO_SN);
    const float3 lpos = f3(v.a.x, v.a.y, v.a.z);
    float3 d = lpos - sd.pos;
    const float dist2 = dot(d, d);
    const float dist = sqrtf(dist2);
    d = d / dist;
    const float3 out_c = sd.to_local(d);
    float3 fc; float fwd_c, rev_c;
    bsdf_eval<LAMBERT>(m, in, out_c, fc, fwd_c, rev_c);
    fc = fc * sd.snc(in, out_c);
    if (all_nonpos(fc)) return f3(0.f);
    fwd_c *= cp; rev_c *= cp;
    SD ls = make_shading(s, v.d.x, v.d.y, __uint_as_float(v.d.z), __uint_as_float(v.d.w), sn);
    const Mat ml = load_material(s, ls.mat, ls.uv);
    if (!(A.flags & S2F_NO_NORMAL_MAPS)) apply_normal_map(s, ls);
    const float3 in_l = ls.to_local(unpack_normal(__float_as_uint(v.c.z)));
    const float3 out_l = ls.to_local(-d);
    float3 fl; float fwd_l, rev_l;
    bsdf_eval<LAMBERT>(ml, in_l, out_l, fl, fwd_l, rev_l);
    fl = fl * snc_adjoint(ls, in_l, out_l);
    if (all_nonpos(fl)) return f3(0.f);
    const float cpl = v.a.w;
    fwd_l *= cpl; rev_l *= cpl;
    const float cam_pdfa = fwd_c * fabsf(out_l.z) / dist2;   // pdfWtoA at the light vertex
    const float light_pdfa = fwd_l * fabsf(out_c.z) / dist2; // pdfWtoA at the camera vertex
    const float w_light = vmis(cam_pdfa) * (A.vm_weight + v.b.w + v.c.x * vmis(rev_l));
    const float w_camera = vmis(light_pdfa) * (A.vm_weight + p.dvcm + p.dvc * vmis(rev_c));
    const float w = vcm_w(A, 1.f / (w_light + 1.f + w_camera));
    const float3 contrib = fc * fl * (w / dist2);
    if (!any_pos(contrib)) return f3(0.f);
    if (vis && !vcm_visible(A, T, ray_offset(sd.pos, sd.gn, d), d, dist * 0.99f)) return f3(0.f);  // AdjustDistance
    return contrib;
}

// GetTargetPdf (vcm.slang:584-608): lum(throughput x pathPdfA x connection) of light vertex v at the
// camera vertex (sd, in, p), 0 outside the path-length range; `c` receives that weighted
// connection.  With `vis` the connection's visibility is traced too, and an occluded one gives 0.
template <bool LAMBERT>
S2D float vcm_lvc_target(const VcmArgs& A, VcmTrace& T, const Mat& m, const SD& sd, float3 in, float cp, const SubPath& p,
                         const LightVertex& v, bool vis, float3& c) {
    c = f3(0.f);
    const uint32_t vlen = __float_as_uint(v.c.w);
    const uint32_t full = vlen + 1 + p.len;
    if (full < A.min_len || full > A.max_len || !vcm_pass(A, p.len + 1, vlen + 1)) return 0.f;
    const float pdfa = v.e.x;
    const float3 thr = f3(v.b.x, v.b.y, v.b.z);
    if (!(pdfa > 0.f) || !any_pos(thr)) return 0.f;
    c = thr * pdfa * vcm_connect<LAMBERT>(A, T, m, sd, in, cp, p, v, vis);
    return luminance(c);
}

// The same target, visibility included, at the camera vertex of a stored reservoir (rebuilt from
// its triangle, as Reuse does with PackedVcmVertex, vcm.slang:647-653).
template <bool LAMBERT>
S2D float vcm_lvc_target_at(const VcmArgs& A, VcmTrace& T, const LvcRecord& q, const LightVertex& v, bool sn) {
    SD sdq = make_shading_local(A.scene, q.instance, q.primitive, q.local_pos, sn);
    const Mat mq = load_material(A.scene, sdq.mat, sdq.uv);
    if (!(A.flags & S2F_NO_NORMAL_MAPS)) apply_normal_map(A.scene, sdq);
    const float3 inq = sdq.to_local(unpack_normal(q.in_dir));
    const float cpq = (A.flags & S2F_NO_RR) ? 1.f : cont_prob(mq);
    SubPath pq;
    pq.thr = f3(1.f);
    pq.dvcm = q.dvcm; pq.dvc = q.dvc; pq.dvm = 0.f;
    pq.fwd_pdfw = 0.f;
    pq.len = q.len;
    pq.specular = false;
    pq.pdfa = 0.f;
    float3 c;
    return vcm_lvc_target<LAMBERT>(A, T, mq, sdq, inq, cpq, pq, v, true, c);
}

// The reuse and the store of ConnectToLVCReservoir (vcm.slang:697-726): updates the reservoir
// (wsum, phat_sel, c_sel, v_sel) in place.
template <bool LAMBERT>
S2D void vcm_lvc_reuse(const VcmArgs& A, VcmTrace& T, const Mat& m, const SD& sd, float3 in, float cp, const SubPath& p,
                       const TravHit& h, float3 dir, Rng& rng, float& wsum, float& phat_sel, float3& c_sel,
                       LightVertex& v_sel) {
    const bool sn = !(A.flags & S2F_NO_SN);
    const uint32_t inst = h.instance, prim = h.primitive;
    const float M = (float)A.lvc_m;
    float Mres = M;
    if (A.lvc_prev_valid) {
        const float4 j = rng.next_float();
        float3 t, b;
        make_orthonormal(sd.gn, t, b);
        const float csz = hg_cell_size(A.lvc_prev, sd.pos);
        const float3 qp = sd.pos + (t * (j.x * 2.f - 1.f) + b * (j.y * 2.f - 1.f)) * csz;
        const uint32_t cell = hg_find_cell<false>(A.lvc_prev, qp, hg_cell_size(A.lvc_prev, qp));
        if (cell != 0xffffffffu) {
            const uint32_t count = A.lvc_prev.cell_counters[cell];
            if (count > 0) {
                const uint32_t off = A.lvc_prev.indices[cell];
                const LvcRecord q = A.lvc_prev_rec[A.lvc_prev.data_indices[off + rng.next().x % count]];
                const float u = rng.next_float().x;
                if (q.M > 0.f) {
                    // target pdfs: q's sample here, and the current sample in q's domain
                    float3 c_new = f3(0.f);
                    const float phat_new = q.W > 0.f && q.phat > 0.f
                                               ? vcm_lvc_target<LAMBERT>(A, T, m, sd, in, cp, p, q.lv, true, c_new) : 0.f;
                    const float phat_i_old = phat_sel > 0.f ? vcm_lvc_target_at<LAMBERT>(A, T, q, v_sel, sn) : 0.f;
                    const float a0 = phat_sel * Mres, b0 = phat_i_old * q.M;
                    const float a1 = q.phat * q.M, b1 = phat_new * Mres;
                    const float m0 = a0 + b0 > 0.f ? a0 / (a0 + b0) : 0.f;
                    const float m1 = a1 + b1 > 0.f ? a1 / (a1 + b1) : 0.f;
                    const float iw0 = phat_sel > 0.f ? wsum / phat_sel : 0.f;
                    Mres += q.M;
                    const float w0 = m0 * phat_sel * iw0;
                    const float w1 = m1 * phat_new * q.W;
                    wsum = w0 + w1;
                    if (u * wsum <= w1) { v_sel = q.lv; phat_sel = phat_new; c_sel = c_new; }
                }
            }
        }
    }
    LvcRecord rec;
    rec.lv = v_sel;
    rec.local_pos = xform_point(A.scene.inv_transforms + 3 * (size_t)inst, sd.pos);
    rec.instance = inst;
    rec.primitive = prim;
    rec.in_dir = pack_normal(-dir);
    rec.len = p.len;
    rec.dvcm = p.dvcm;
    rec.dvc = p.dvc;
    rec.M = fminf(Mres, A.lvc_max_m * M);
    rec.W = phat_sel > 0.f ? wsum / phat_sel : 0.f;
    rec.phat = phat_sel;
    ReservoirRecord key;  // what the grid build sorts a cell's records by
    key.local_pos = rec.local_pos;
    key.instance = inst;
    key.rnd = make_float4(v_sel.a.x, v_sel.a.y, v_sel.a.z, v_sel.b.x);
    key.target_pdf = rec.phat;
    key.W = rec.W;
    key.M = rec.M;
    key.primitive = prim;
    key.local_dir_in = f3(0.f);
    key.pad = 0.f;
    const uint32_t idx = hg_append(A.lvc_cur, sd.pos, key);
    if (idx != 0xffffffffu) A.lvc_cur_rec[idx] = rec;
}

// ConnectToLVCReservoir (vcm.slang:568-736): lvc_m cached light vertices picked at random,
// resampled by the target above with source pdf pathPdfA (the discrete pick's 1 / count cancels in
// the estimate), one shadow ray for the chosen one.  With reuse (S2_VCM_FLAG_LVC_REUSE) a reservoir
// of the previous iteration found in the hash grid near the vertex is resampled in with the
// pairwise MIS weights of Reuse (vcm.slang:633-678), and this vertex's reservoir is stored for the
// next iteration: every one, also those of weight 0, as with the direct-illumination reservoirs (a
// population of successes only would be conditional on success and too bright).  Returns the
// contribution to add with the camera throughput, already scaled by cached vertices / light
// subpaths.  (h, dir): the camera vertex's hit and the ray that reached it.  Out of line: inlined,
// the reservoir state spills in the camera kernel.
template <bool LAMBERT>
__device__ __noinline__ float3 vcm_connect_lvc_ris(const VcmArgs& A, VcmTrace& T, const Mat& m, const SD& sd, float3 in, float cp,
                               const SubPath& p, uint32_t total, const TravHit& h, float3 dir, Rng& rng) {
    float wsum = 0.f, phat_sel = 0.f;
    float3 c_sel = f3(0.f);
    LightVertex v_sel;
    v_sel.a = v_sel.b = v_sel.c = v_sel.e = make_float4(0.f, 0.f, 0.f, 0.f);
    v_sel.d = make_uint4(0u, 0u, 0u, 0u);
    const float M = (float)A.lvc_m;
    for (uint32_t i = 0; i < A.lvc_m; ++i) {
        const LightVertex v = A.lv[A.lvc_list[rng.next().x % total]];
        const float u = rng.next_float().x;
        float3 c;
        const float phat = vcm_lvc_target<LAMBERT>(A, T, m, sd, in, cp, p, v, false, c);
        if (!(phat > 0.f)) continue;
        const float wi = phat / (v.e.x * M);
        wsum += wi;
        if (u * wsum <= wi) { phat_sel = phat; c_sel = c; v_sel = v; }
    }
    if (phat_sel > 0.f) {
        const float3 lpos = f3(v_sel.a.x, v_sel.a.y, v_sel.a.z);
        float3 d = lpos - sd.pos;
        const float dist = length(d);
        d = d / dist;
        if (!vcm_visible(A, T, ray_offset(sd.pos, sd.gn, d), d, dist * 0.99f)) phat_sel = 0.f;
    }
    if (A.lvc_reuse)
        vcm_lvc_reuse<LAMBERT>(A, T, m, sd, in, cp, p, h, dir, rng, wsum, phat_sel, c_sel, v_sel);
    if (!(phat_sel > 0.f)) return f3(0.f);
    return c_sel * ((wsum / phat_sel) * ((float)total / (float)A.n_light));
}

// ProcessVertex (vcm.slang:842-875): merging with one light vertex, MIS of tech. rep. eqs. 37-39.
// The merged estimate uses the camera BSDF value without the cosine that evaluateReflectance carries
// (the light vertex density already holds the projected area), as SmallVCM's ProcessVertex does.
template <bool LAMBERT>
S2D float3 vcm_merge_one(const VcmArgs& A, const Mat& m, const SD& sd, float3 in, float cp, const SubPath& p,
                         const LightVertex& v) {
    const uint32_t vlen = __float_as_uint(v.c.w);
    if (vlen + p.len > A.max_len || vlen + p.len < A.min_len) return f3(0.f);
    if (!vcm_pass(A, p.len + 1, vlen)) return f3(0.f);
    const float3 out = sd.to_local(unpack_normal(__float_as_uint(v.c.z)));
    float3 f; float fwd, rev;
    bsdf_eval<LAMBERT>(m, in, out, f, fwd, rev);
    f = f * sd.snc(in, out);
    if (all_nonpos(f) || !(fabsf(out.z) > 0.f)) return f3(0.f);
    fwd *= cp;
    rev *= v.a.w;  // the light vertex's continuation probability governs the reverse direction
    const float w_light = v.b.w * A.vc_weight + v.c.y * vmis(fwd);
    const float w_camera = p.dvcm * A.vc_weight + p.dvm * vmis(rev);
    const float w = A.ppm ? 1.f : vcm_w(A, 1.f / (w_light + 1.f + w_camera));
    return f * f3(v.b.x, v.b.y, v.b.z) * (w * A.vm_norm / fabsf(out.z));
}

// MergeVertices (vcm.slang:801-840): the 2x2x2 cells nearest the query; buckets holding more than
// 64 vertices are subsampled 64 times with weight count / 64.
template <bool LAMBERT>
S2D float3 vcm_merge(const VcmArgs& A, const Mat& m, const SD& sd, float3 in, float cp, const SubPath& p, Rng& rng) {
    const float3 q = sd.pos;
    const float r2 = A.merge_radius * A.merge_radius;
    const float3 g = f3(q.x / A.cell_size, q.y / A.cell_size, q.z / A.cell_size);
    const int3 c0 = make_int3((int)floorf(g.x), (int)floorf(g.y), (int)floorf(g.z));
    const int sx = (g.x - floorf(g.x)) < 0.5f ? -1 : 1, sy = (g.y - floorf(g.y)) < 0.5f ? -1 : 1,
              sz = (g.z - floorf(g.z)) < 0.5f ? -1 : 1;
    float3 sum = f3(0.f);
    for (int j = 0; j < 8; ++j) {
        const int3 c = make_int3(c0.x + (j & 1) * sx, c0.y + ((j >> 1) & 1) * sy, c0.z + (j >> 2) * sz);
        const uint32_t bucket = vcm_cell_hash(c) & A.grid_mask;
        const uint32_t start = A.grid_start[bucket], end = A.grid_end[bucket];
        const uint32_t cnt = end - start;
        if (cnt == 0) continue;
        const uint32_t n = min(cnt, 64u);
        const float wsub = cnt > 64u ? (float)cnt / 64.f : 1.f;
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t k = cnt > 64u ? rng.next().x % cnt : i;
            const LightVertex v = A.lv[A.grid_slot[start + k]];
            const float3 vp = f3(v.a.x, v.a.y, v.a.z);
            const int3 vc = vcm_cell(A, vp);
            if (vc.x != c.x || vc.y != c.y || vc.z != c.z) continue;  // another cell in the same bucket
            const float3 dq = vp - q;
            if (dot(dq, dq) > r2) continue;
            sum = sum + vcm_merge_one<LAMBERT>(A, m, sd, in, cp, p, v) * wsub;
        }
    }
    return sum;
}

// ---------------------------------------------------------------- direct-illumination reservoirs
// ReservoirStateDI (vcm.slang:251-340): resampled light samples with the target pdf
// lum(Le) |n_s . w| G, no BSDF.  A sample is its four random numbers; `r` receives it evaluated at
// (pos, ns).  GetTargetPdf<true> also traces the sample's visibility from (pos, gn).
S2D float vcm_di_target(const VcmArgs& A, VcmTrace& T, float3 pos, float3 ns, float3 gn, float4 x, bool sn, bool vis,
                        Illum& r) {
    r = sample_illum(A.scene, x, pos, sn);
    if (!(r.pdf > 0.f) || !any_pos(r.radiance)) return 0.f;
    const float g = r.finite ? r.cos_light / (r.dist * r.dist) : 1.f;
    const float t = luminance(r.radiance) * fabsf(dot(ns, r.dir)) * g;
    if (vis && t > 0.f && !vcm_visible(A, T, ray_offset(pos, gn, r.dir), r.dir, r.dist * 0.99f)) return 0.f;
    return t;
}

struct VcmReservoir {
    float4 rnd;      // the selected sample
    Illum r;         // it, evaluated at the camera vertex
    float phat;      // its target pdf (0 when occluded)
    float wsum;      // total resampling weight
    float M;
    S2D float iw() const { return phat > 0.f ? wsum / phat : 0.f; }  // mIntegrationWeight
};

// Reuse (vcm.slang:296-340): resamples the stored reservoir q into `res` with the pairwise MIS
// weights over the two domains' visibility-aware target pdfs.
S2D void vcm_di_reuse(const VcmArgs& A, VcmTrace& T, const SD& sd, const ReservoirRecord& q, VcmReservoir& res, Rng& rng,
                      bool sn) {
    if (!(q.M > 0.f)) return;
    const SD sdq = make_shading_local(A.scene, q.instance, q.primitive, q.local_pos, sn);
    Illum tmp, nr;
    const float phat_i_old = vcm_di_target(A, T, sdq.pos, sdq.n, sdq.gn, res.rnd, sn, true, tmp);  // current sample, q's domain
    const float phat_new = vcm_di_target(A, T, sd.pos, sd.n, sd.gn, q.rnd, sn, true, nr);           // q's sample, this domain
    const float a0 = res.phat * res.M, b0 = phat_i_old * q.M;
    const float a1 = q.target_pdf * q.M, b1 = phat_new * res.M;
    const float m0 = a0 + b0 > 0.f ? a0 / (a0 + b0) : 0.f;
    const float m1 = a1 + b1 > 0.f ? a1 / (a1 + b1) : 0.f;
    const float iw0 = res.iw();
    res.M += q.M;
    const float w0 = m0 * res.phat * iw0;
    const float w1 = m1 * phat_new * q.W;
    res.wsum = w0 + w1;
    if (rng.next_float().x * res.wsum <= w1) {
        res.rnd = q.rnd;
        res.phat = phat_new;
        res.r = nr;
    }
}

// SampleDirectIlluminationReservoir (vcm.slang:343-390): di_m candidates, the chosen one's shadow
// ray, optionally the reuse of a previous reservoir found near the vertex, and the store of this
// one (whatever its weight, see below).  Returns the reservoir (integration weight iw(); its
// sample in r).
S2D VcmReservoir vcm_di_reservoir(const VcmArgs& A, VcmTrace& T, const SD& sd, uint32_t inst, uint32_t prim, Rng& rng,
                                  bool sn) {
    VcmReservoir res;
    res.rnd = make_float4(0.f, 0.f, 0.f, 0.f);
    res.phat = 0.f; res.wsum = 0.f; res.M = (float)A.di_m;
    res.r.radiance = f3(0.f); res.r.pdf = 0.f; res.r.dir = f3(0.f); res.r.dist = 0.f; res.r.cos_light = 0.f; res.r.finite = true;
    for (uint32_t c = 0; c < A.di_m; ++c) {  // ProcessSample
        const float4 x = rng.next_float();
        const float u = rng.next_float().x;
        Illum r;
        const float phat = vcm_di_target(A, T, sd.pos, sd.n, sd.gn, x, sn, false, r);
        if (!(phat > 0.f)) continue;
        const float wi = phat / (r.pdf * res.M);
        res.wsum += wi;
        if (u * res.wsum <= wi) { res.rnd = x; res.phat = phat; res.r = r; }
    }
    if (res.phat > 0.f && !vcm_visible(A, T, ray_offset(sd.pos, sd.gn, res.r.dir), res.r.dir, res.r.dist * 0.99f))
        res.phat = 0.f;
    if (A.di_reuse) {
        if (A.di_prev_valid) {
            const float4 j = rng.next_float();
            float3 t, b;
            make_orthonormal(sd.gn, t, b);
            const float csz = hg_cell_size(A.di_prev, sd.pos);
            const float3 qp = sd.pos + (t * (j.x * 2.f - 1.f) + b * (j.y * 2.f - 1.f)) * csz;
            const uint32_t cell = hg_find_cell<false>(A.di_prev, qp, hg_cell_size(A.di_prev, qp));
            if (cell != 0xffffffffu) {
                const uint32_t count = A.di_prev.cell_counters[cell];
                if (count > 0) {
                    const uint32_t off = A.di_prev.indices[cell];
                    const ReservoirRecord q = A.di_prev.data[A.di_prev.data_indices[off + rng.next().x % count]];
                    vcm_di_reuse(A, T, sd, q, res, rng, sn);
                }
            }
        }
        // Every reservoir is stored, also those of integration weight 0 (no candidate, or the chosen
        // one occluded).  The reference appends only positive weights (vcm.slang:370), which makes
        // the reused population conditional on success: its expected weight is then 1 / P(W > 0)
        // too large, and on the box scene the image came out 3.9 % too bright.
        {
            ReservoirRecord rec;
            rec.local_pos = xform_point(A.scene.inv_transforms + 3 * (size_t)inst, sd.pos);
            rec.instance = inst;
            rec.primitive = prim;
            rec.rnd = res.rnd;
            rec.target_pdf = res.phat;
            rec.W = res.iw();
            rec.M = fminf(res.M, A.di_max_m * (float)A.di_m);
            rec.local_dir_in = f3(0.f);
            rec.pad = 0.f;
            hg_append(A.di_cur, sd.pos, rec);
        }
    }
    return res;
}

// LVC_RIS: the variant for the light-vertex-cache reservoirs (lvc_m > 0), compiled apart so that
// the other techniques' code keeps its registers.
template <bool LAMBERT, bool LVC_RIS>
__global__ void __launch_bounds__(128) k_vcm_camera(const __grid_constant__ VcmArgs A) {
    __shared__ uint2 stack[S2_STACK_SMEM * 128];
    VcmTrace T{stack + threadIdx.x, 128u, 0u, 0u, false, {0, 0}};
    const DevScene& s = A.scene;
    const bool sn = !(A.flags & S2F_NO_SN);
    const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix < A.pixels) {
        const uint32_t px = pix % A.width, py = pix / A.width;
        Rng rng = make_rng(px, py, A.seed, (A.flags & S2F_PCG32) != 0);
        // GenerateCameraSample (vcm.slang:140-173), with the pixel position jittered over the pixel
        // so that camera paths and camera connections integrate the same box pixel filter
        const float4 j = rng.next_float();
        float3 dir = camera_dir(A.proj, A.imin, A.imax, A.cam, px, py, j.x, j.y);
        const float* ci = A.cam_inv;
        const float dcz = ci[8] * dir.x + ci[9] * dir.y + ci[10] * dir.z;
        const float cos_cam = fabsf(dcz);
        const float ipd = A.image_plane_dist / cos_cam;
        const float camera_pdfw = ipd * ipd / cos_cam;
        float3 org = f3(A.cam[3], A.cam[7], A.cam[11]);
        SubPath p;
        p.thr = f3(1.f);
        p.dvcm = vmis((float)A.n_light / camera_pdfw);
        p.dvc = p.dvm = 0.f;
        p.fwd_pdfw = S2_INF;
        p.len = 1;
        p.specular = true;
        float3 L = f3(0.f);
        while (true) {
            const TravHit h = vcm_closest(A, T, org, dir);
            if (h.tri == 0xffffffffu) {
                if (p.len == 1 && A.write_aovs) {
                    if (A.aov_albedo) A.aov_albedo[pix] = make_float4(0.f, 0.f, 0.f, 1.f);  // VCM: miss albedo 0
                    if (A.aov_vis) A.aov_vis[pix] = make_uint2(0xffffffffu, pack_normal(dir));
                    if (A.aov_depth) A.aov_depth[pix] = make_float4(S2_INF, S2_INF, 1.f, 1.f);
                    if (A.aov_prev_uv) A.aov_prev_uv[pix] = make_float2(((float)px + 0.5f) / (float)A.width, ((float)py + 0.5f) / (float)A.height);
                    if (A.aov_ids) A.aov_ids[pix] = make_uint2(0xffffffffu, 0xffffffffu);
                }
                break;  // the environment is black in this renderer
            }
            SD sd = make_shading(s, h.instance, h.primitive, h.b1, h.b2, sn);
            const Mat m = load_material(s, sd.mat, sd.uv);
            if (!(A.flags & S2F_NO_NORMAL_MAPS)) apply_normal_map(s, sd);
            const float3 in = sd.to_local(-dir);
            if (p.len == 1 && A.write_aovs) {  // StoreAuxillaryData (vcm.slang:176-198)
                const float3 bc = m.base();
                if (A.aov_albedo) A.aov_albedo[pix] = make_float4(bc.x, bc.y, bc.z, 1.f);
                if (A.aov_vis) A.aov_vis[pix] = make_uint2((h.instance & 0xffffu) | (h.primitive << 16), sd.ns);
                if (A.aov_ids) A.aov_ids[pix] = make_uint2(h.instance, h.primitive);
                const float3 pw = xform_point(s.motion_transforms + 3 * (size_t)h.instance, sd.pos);
                const float3 pc = prev_camera_point(A.prev_inv, pw);
                float2 pr = make_float2((float)px + 0.5f, (float)py + 0.5f);
                camera_to_raster(A.proj, A.imin, A.imax, pc, pr);
                if (A.aov_prev_uv) A.aov_prev_uv[pix] = make_float2(pr.x / (float)A.width, pr.y / (float)A.height);
                if (A.aov_depth) A.aov_depth[pix] = make_float4(h.t, length(pc), 1.f, 1.f);
            }
            // tech. rep. eqs. 31-36, completed at the hit
            const float cos_in = fabsf(in.z);
            p.dvcm *= vmis(h.t * h.t);
            p.dvcm /= vmis(cos_in);
            p.dvc /= vmis(cos_in);
            p.dvm /= vmis(cos_in);
            const float fwd_g = cos_in / (h.t * h.t);
            // GetSurfaceRadiance + GetLightRadiance (vcm.hlsli:314-329, vcm.slang:209-244): lights do
            // not reflect, so the path ends at an emitter seen from its emitting side
            const float cos_e = -dot(dir, sd.gn);
            if (any_pos(m.emission()) && cos_e >= 0.f && s.light_count > 0) {
                if (p.len >= A.min_len && vcm_pass(A, p.len + 1, 0)) {
                    float w = 1.f;
                    if (p.len > 1) {
                        const float direct_pdfa = light_pdfa(s, h.instance, sd.area);
                        const float emission_pdfw = direct_pdfa * cos_hemisphere_pdfw(cos_e);
                        if (A.use_vm && !A.use_vc) w = p.specular ? 1.f : 0.f;
                        else if (A.path_trace_only) w = vcm_w(A, 1.f / (1.f + vmis(direct_pdfa / fwd_g) / vmis(p.fwd_pdfw)));
                        else w = vcm_w(A, 1.f / (1.f + vmis(direct_pdfa) * p.dvcm + vmis(emission_pdfw) * p.dvc));
                    }
                    L = L + p.thr * m.emission() * w;
                }
                break;
            }
            if (!any_pos(m.base())) break;
            if (p.len >= A.max_len) break;
            const bool sing = mat_singular<LAMBERT>(m);
            const float cp = (A.flags & S2F_NO_RR) ? 1.f : cont_prob(m);
            if (!sing) {
                // DirectIllumination (vcm.slang:396-475): MIS of tech. rep. eqs. 37, 44-45
                if ((A.use_vc || A.path_trace_only) && p.len + 1 >= A.min_len) {
                    // the light sample: resampled (visibility traced inside) or one sample (its
                    // shadow ray below); iw: its contribution weight per unit area
                    Illum r;
                    float iw;
                    if (A.di_ris) {
                        const VcmReservoir res = vcm_di_reservoir(A, T, sd, h.instance, h.primitive, rng, sn);
                        r = res.r;
                        iw = res.iw();
                    } else {
                        r = sample_illum(s, rng.next_float(), sd.pos, sn);
                        iw = r.pdf > 0.f ? 1.f / r.pdf : 0.f;
                    }
                    if (any_pos(r.radiance) && r.pdf > 0.f && iw > 0.f && vcm_pass(A, p.len + 1, 1)) {
                        const float direct_pdfw = r.pdf * r.dist * r.dist / r.cos_light;
                        const float emission_pdfw = r.pdf * cos_hemisphere_pdfw(r.cos_light);
                        const float3 out = sd.to_local(r.dir);
                        float3 f; float fwd, rev;
                        bsdf_eval<LAMBERT>(m, in, out, f, fwd, rev);
                        f = f * sd.snc(in, out);
                        if (any_pos(f)) {
                            const float bsdf_dir = fwd * cp, bsdf_rev = rev * cp;
                            float w;
                            if (A.path_trace_only) {
                                w = vcm_w(A, 1.f / (1.f + vmis(bsdf_dir) / vmis(direct_pdfw)));
                            } else {
                                const float w_light = vmis(bsdf_dir / direct_pdfw);
                                const float w_camera = vmis(emission_pdfw * fabsf(out.z) / (direct_pdfw * r.cos_light)) *
                                                       (A.vm_weight + p.dvcm + p.dvc * vmis(bsdf_rev));
                                w = vcm_w(A, 1.f / (w_light + 1.f + w_camera));
                            }
                            // 1 / direct_pdfw without resampling; iw G with it (vcm.slang:390, 463)
                            const float g = r.cos_light / (r.dist * r.dist);
                            const float3 contrib = r.radiance * f * (A.di_ris ? w * iw * g : w / direct_pdfw);
                            if (any_pos(contrib) &&
                                (A.di_ris || vcm_visible(A, T, ray_offset(sd.pos, sd.gn, r.dir), r.dir, r.dist * 0.99f)))
                                L = L + p.thr * contrib;
                        }
                    }
                }
                if (!A.path_trace_only) {
                    if (LVC_RIS && A.use_vc && A.lvc && A.lvc_total) {
                        const uint32_t total = *A.lvc_total;
                        if (total > 0)
                            L = L + p.thr * vcm_connect_lvc_ris<LAMBERT>(A, T, m, sd, in, cp, p, total, h, dir, rng);
                    } else if (A.use_vc && A.lvc && A.lvc_total) {
                        // ConnectToLVC (vcm.slang:732-753): one random cached vertex, weighted by the
                        // cached vertex count over the light subpath count
                        const uint32_t total = *A.lvc_total;
                        if (total > 0) {
                            const uint32_t idx = rng.next().x % total;
                            const LightVertex v = A.lv[A.lvc_list[idx]];
                            const uint32_t vlen = __float_as_uint(v.c.w);
                            const uint32_t full = vlen + 1 + p.len;
                            if (full >= A.min_len && full <= A.max_len && vcm_pass(A, p.len + 1, vlen + 1))
                                L = L + p.thr * f3(v.b.x, v.b.y, v.b.z) * vcm_connect<LAMBERT>(A, T, m, sd, in, cp, p, v) *
                                            ((float)total / (float)A.n_light);
                        }
                    } else if (A.use_vc) {
                        // ConnectToLightPath (vcm.slang:756-784): every vertex of light subpath pix mod n
                        const uint32_t lp = pix % A.n_light;
                        const uint32_t cnt = A.lv_count[lp];
                        for (uint32_t k = 0; k < cnt; ++k) {
                            const LightVertex v = A.lv[(size_t)k * A.n_light + lp];
                            const uint32_t vlen = __float_as_uint(v.c.w);
                            const uint32_t full = vlen + 1 + p.len;
                            if (full < A.min_len || !any_pos(f3(v.b.x, v.b.y, v.b.z))) continue;
                            if (full > A.max_len) break;  // stored in increasing length
                            if (!vcm_pass(A, p.len + 1, vlen + 1)) continue;
                            L = L + p.thr * f3(v.b.x, v.b.y, v.b.z) * vcm_connect<LAMBERT>(A, T, m, sd, in, cp, p, v);
                        }
                    }
                    if (A.use_vm && A.grid_start) {
                        L = L + p.thr * vcm_merge<LAMBERT>(A, m, sd, in, cp, p, rng);
                        if (A.ppm) break;  // PPM merges at the first non-singular camera vertex only
                    }
                }
            }
            if (!vcm_scatter<LAMBERT, false>(A, m, sd, in, sing, rng, p, dir)) break;
            org = ray_offset(sd.pos, sd.gn, dir);
            p.len++;
        }
        vcm_splat(A, pix, L);
    }
    for (int o = 16; o > 0; o >>= 1) { T.ext += __shfl_xor_sync(0xffffffffu, T.ext, o); T.shadow += __shfl_xor_sync(0xffffffffu, T.shadow, o); }
    if ((threadIdx.x & 31u) == 0) { atomicAdd(A.counts, (unsigned long long)T.ext); atomicAdd(A.counts + 1, (unsigned long long)T.shadow); }
    if (T.overflow) atomicOr(A.status, 1);
}

}  // namespace s2
