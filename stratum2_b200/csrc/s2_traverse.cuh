// BVH8 traversal for closest-hit and first-hit queries.
//
// Replaces the hardware RayQuery loop of the reference (src/Shaders/common/intersection.hlsli:
// 68-193, traceRay; :262-338, traceVisibilityRay without media).  Semantics kept from the
// reference: a hit is accepted for tmin <= t <= tmax (RayDesc TMin/TMax); a first-hit query
// (RAY_FLAG_ACCEPT_FIRST_HIT_AND_END_SEARCH) stops at the first accepted triangle.  Added here:
// closest-hit ties (equal t) resolve to the lowest (instance, primitive) so results do not depend
// on traversal order.
//
// Triangle test: watertight ray/triangle intersection (Woop, Benthin and Wald, JCGT 2013) with
// the double-precision fallback for zero edge functions.  Every float operation uses an explicit
// round-to-nearest intrinsic so the compiler cannot contract it into an FMA: the result is then
// bit-identical to a CPU evaluation of the same operations in IEEE single precision.
#pragma once
#include "s2_bvh.h"
#include "s2_math.cuh"

struct TravRay {
    float3 o, d;
    float3 inv_d;
    float tmin;
    uint32_t oct;       // bit i set when d[i] < 0
    int kx, ky, kz;     // watertight axis permutation
    float Sx, Sy, Sz;   // shear constants
};

S2D float safe_inv(float d) {
    // avoid 0*inf = NaN in the slab test for axis-parallel rays
    const float dd = fabsf(d) < 1e-30f ? copysignf(1e-30f, d) : d;
    return __fdiv_rn(1.f, dd);
}

S2D float comp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

S2D TravRay make_trav_ray(float3 o, float3 d, float tmin) {
    TravRay r;
    r.o = o; r.d = d; r.tmin = tmin;
    r.inv_d = f3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
    r.oct = (d.x < 0 ? 1u : 0u) | (d.y < 0 ? 2u : 0u) | (d.z < 0 ? 4u : 0u);
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = (ax > ay) ? ((ax > az) ? 0 : 2) : ((ay > az) ? 1 : 2);
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    if (comp(d, kz) < 0.f) { const int t = kx; kx = ky; ky = t; }
    r.kx = kx; r.ky = ky; r.kz = kz;
    const float dz = comp(d, kz);
    r.Sx = __fdiv_rn(comp(d, kx), dz);
    r.Sy = __fdiv_rn(comp(d, ky), dz);
    r.Sz = __fdiv_rn(1.f, dz);
    return r;
}

// Watertight triangle test.  Returns true and sets t, b1, b2 when the triangle is hit with
// tmin <= t <= tmax.
S2D bool intersect_triangle(const TravRay& r, float3 v0, float3 v1, float3 v2, float tmax, float& t_out, float& b1, float& b2) {
    const float3 A = f3(__fsub_rn(v0.x, r.o.x), __fsub_rn(v0.y, r.o.y), __fsub_rn(v0.z, r.o.z));
    const float3 B = f3(__fsub_rn(v1.x, r.o.x), __fsub_rn(v1.y, r.o.y), __fsub_rn(v1.z, r.o.z));
    const float3 C = f3(__fsub_rn(v2.x, r.o.x), __fsub_rn(v2.y, r.o.y), __fsub_rn(v2.z, r.o.z));
    const float Akz = comp(A, r.kz), Bkz = comp(B, r.kz), Ckz = comp(C, r.kz);
    const float Ax = __fsub_rn(comp(A, r.kx), __fmul_rn(r.Sx, Akz));
    const float Ay = __fsub_rn(comp(A, r.ky), __fmul_rn(r.Sy, Akz));
    const float Bx = __fsub_rn(comp(B, r.kx), __fmul_rn(r.Sx, Bkz));
    const float By = __fsub_rn(comp(B, r.ky), __fmul_rn(r.Sy, Bkz));
    const float Cx = __fsub_rn(comp(C, r.kx), __fmul_rn(r.Sx, Ckz));
    const float Cy = __fsub_rn(comp(C, r.ky), __fmul_rn(r.Sy, Ckz));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.f || V == 0.f || W == 0.f) {
        U = (float)__dsub_rn(__dmul_rn((double)Cx, (double)By), __dmul_rn((double)Cy, (double)Bx));
        V = (float)__dsub_rn(__dmul_rn((double)Ax, (double)Cy), __dmul_rn((double)Ay, (double)Cx));
        W = (float)__dsub_rn(__dmul_rn((double)Bx, (double)Ay), __dmul_rn((double)By, (double)Ax));
    }
    if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return false;
    const float det = __fadd_rn(__fadd_rn(U, V), W);
    if (det == 0.f) return false;
    const float Az = __fmul_rn(r.Sz, Akz), Bz = __fmul_rn(r.Sz, Bkz), Cz = __fmul_rn(r.Sz, Ckz);
    const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
    const float t = __fdiv_rn(T, det);
    if (!(t >= r.tmin && t <= tmax)) return false;
    t_out = t;
    b1 = __fdiv_rn(V, det);
    b2 = __fdiv_rn(W, det);
    return true;
}

struct TravHit {
    float t;
    uint32_t tri;        // triangle record index (BVH order), 0xffffffff when missed
    uint32_t instance, primitive;
    float b1, b2;
};

struct TravCounters { uint32_t nodes, tris; };

S2D uint32_t extract_byte(uint32_t w, uint32_t i) { return (w >> (8 * i)) & 0xffu; }

// Byte i of w as a float.  The node test spreads the 48 conversions of a node over two pipes:
// x planes by integer-to-float conversion, y and z planes through the mantissa (2^23 + b is
// exact, and so is the subtraction), measured 2.4 % faster on B200 than converting all six.
S2D float byte_f_prmt(uint32_t w, uint32_t i) {
    return __uint_as_float(__byte_perm(w, 0x4Bu, i | 0x4550u)) - 8388608.f;
}
S2D float byte_f_cvt(uint32_t w, uint32_t i) { return (float)extract_byte(w, i); }
// three-input min / max (sm_100)
S2D float max3f(float a, float b, float c) {
    float d; asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c)); return d;
}
S2D float min3f(float a, float b, float c) {
    float d; asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c)); return d;
}

// Intersect the 8 children of `node` with [tmin, tmax].  Returns the hit mask in bit-position
// space (bit b = slot b ^ oct) for internal children, and the triangle mask for leaf slots.
S2D void intersect_node(const TravRay& r, const uint4* __restrict__ nodes4, uint32_t node_idx, float tmax,
                        uint32_t& child_base, uint32_t& imask, uint32_t& hits, uint32_t& tri_base, uint32_t& trimask) {
    const uint4* np = nodes4 + (size_t)node_idx * 8;  // 128-byte stride
    const uint4 n0 = __ldg(np + 0);
    const uint4 n1 = __ldg(np + 1);
    const uint4 n2 = __ldg(np + 2);
    const uint4 n3 = __ldg(np + 3);
    const uint4 n4 = __ldg(np + 4);
    const float px = __uint_as_float(n0.x), py = __uint_as_float(n0.y), pz = __uint_as_float(n0.z);
    const uint32_t ex = n0.w & 0xffu, ey = (n0.w >> 8) & 0xffu, ez = (n0.w >> 16) & 0xffu;
    imask = n0.w >> 24;
    child_base = n1.x;
    tri_base = n1.y;
    const uint32_t meta_lo = n1.z, meta_hi = n1.w;
    const float sx = __uint_as_float(ex << 23) * r.inv_d.x;
    const float sy = __uint_as_float(ey << 23) * r.inv_d.y;
    const float sz = __uint_as_float(ez << 23) * r.inv_d.z;
    const float ax = (px - r.o.x) * r.inv_d.x;
    const float ay = (py - r.o.y) * r.inv_d.y;
    const float az = (pz - r.o.z) * r.inv_d.z;
    // near/far plane bytes per axis, swapped for negative directions
    const uint32_t xlo0 = n2.x, xlo1 = n2.y, ylo0 = n2.z, ylo1 = n2.w;
    const uint32_t zlo0 = n3.x, zlo1 = n3.y, xhi0 = n3.z, xhi1 = n3.w;
    const uint32_t yhi0 = n4.x, yhi1 = n4.y, zhi0 = n4.z, zhi1 = n4.w;
    const bool nx = r.inv_d.x < 0, ny = r.inv_d.y < 0, nz = r.inv_d.z < 0;
    const uint32_t xn0 = nx ? xhi0 : xlo0, xn1 = nx ? xhi1 : xlo1, xf0 = nx ? xlo0 : xhi0, xf1 = nx ? xlo1 : xhi1;
    const uint32_t yn0 = ny ? yhi0 : ylo0, yn1 = ny ? yhi1 : ylo1, yf0 = ny ? ylo0 : yhi0, yf1 = ny ? ylo1 : yhi1;
    const uint32_t zn0 = nz ? zhi0 : zlo0, zn1 = nz ? zhi1 : zlo1, zf0 = nz ? zlo0 : zhi0, zf1 = nz ? zlo1 : zhi1;
    uint32_t m = 0;  // children whose box the ray segment overlaps, in slot order
#pragma unroll
    for (uint32_t s = 0; s < 8; ++s) {
        const uint32_t w = s < 4 ? 0 : 1, i = s & 3;
        const float qnx = byte_f_cvt(w ? xn1 : xn0, i), qfx = byte_f_cvt(w ? xf1 : xf0, i);
        const float qny = byte_f_prmt(w ? yn1 : yn0, i), qfy = byte_f_prmt(w ? yf1 : yf0, i);
        const float qnz = byte_f_prmt(w ? zn1 : zn0, i), qfz = byte_f_prmt(w ? zf1 : zf0, i);
        const float tnx = fmaf(qnx, sx, ax), tfx = fmaf(qfx, sx, ax);
        const float tny = fmaf(qny, sy, ay), tfy = fmaf(qfy, sy, ay);
        const float tnz = fmaf(qnz, sz, az), tfz = fmaf(qfz, sz, az);
        // min(tf, tmax) * c == min(tf * c, tmax * c): the padding also covers tmax
        const float tn = max3f(tnx, tny, fmaxf(tnz, r.tmin));
        const float tf = min3f(tfx, tfy, fminf(tfz, tmax)) * 1.0000004f;
        if (tn <= tf) m |= 1u << s;
    }
    // internal children: bit s ^ oct (the octant order), by three conditional swaps of bit groups
    uint32_t h = m & imask;
    if (r.oct & 1u) h = ((h & 0x55u) << 1) | ((h >> 1) & 0x55u);
    if (r.oct & 2u) h = ((h & 0x33u) << 2) | ((h >> 2) & 0x33u);
    if (r.oct & 4u) h = ((h & 0x0fu) << 4) | ((h >> 4) & 0x0fu);
    hits = h;
    // leaf children: their triangle ranges (usually one or two per node)
    trimask = 0;
    uint32_t leaf = m & ~imask & 0xffu;
    while (leaf) {
        const uint32_t s = __ffs(leaf) - 1;
        leaf &= leaf - 1;
        const uint32_t meta = extract_byte(s < 4 ? meta_lo : meta_hi, s & 3u);
        trimask |= ((1u << (meta >> 5)) - 1u) << (meta & 31u);
    }
}

// Per-ray traversal state for the step-wise traversal: the current node, the stack pointer and
// the closest hit so far.  The stack lives in shared memory (first S2_STACK_SMEM entries, strided
// by `lane_stride`) and in a local-memory continuation `lstack`.
// Alpha test of a candidate hit (closest or any hit); NoAlphaTest accepts every triangle.
struct NoAlphaTest {
    S2D bool operator()(uint32_t, uint32_t, float, float) const { return true; }
};

struct TravState {
    uint32_t node;
    int sp;
    bool ok;    // false if the stack overflowed
    uint32_t tbase, tmask;  // pending leaf triangles (trav_step_pp)
};

S2D void trav_begin(TravState& st, TravHit& hit, float tmax) {
    st.node = 0; st.sp = 0; st.ok = true; st.tbase = 0; st.tmask = 0;
    hit.t = tmax; hit.tri = 0xffffffffu; hit.instance = 0xffffffffu; hit.primitive = 0xffffffffu;
    hit.b1 = hit.b2 = 0.f;
}

// One traversal step: visit st.node (its 8 child boxes and its leaf triangles), then choose the
// next node (nearest hit child, else the stack).  Returns true when the traversal is finished.
// Triangles flagged S2_TRI_ALPHA_TESTED are accepted only when `alpha(instance, primitive, b1, b2)`.
template <bool ANYHIT, bool COUNT, class Alpha = NoAlphaTest>
S2D bool trav_step(const TravRay& r, TravState& st, const uint4* __restrict__ nodes4, const float4* __restrict__ tris4,
                   uint2* __restrict__ smem_stack, uint32_t lane_stride, uint2* lstack, TravHit& hit, TravCounters& ctr,
                   const Alpha& alpha = Alpha()) {
    uint32_t child_base, imask, hits, tri_base, trimask;
    intersect_node(r, nodes4, st.node, hit.t, child_base, imask, hits, tri_base, trimask);
    if (COUNT) ctr.nodes++;
    while (trimask) {
        const uint32_t k = __ffs(trimask) - 1;
        trimask &= trimask - 1;
        const uint32_t ti = tri_base + k;
        const float4 a = __ldg(tris4 + 3 * (size_t)ti + 0);
        const float4 b = __ldg(tris4 + 3 * (size_t)ti + 1);
        const float4 c = __ldg(tris4 + 3 * (size_t)ti + 2);
        if (COUNT) ctr.tris++;
        float t, b1, b2;
        if (intersect_triangle(r, ld3(a), ld3(b), ld3(c), hit.t, t, b1, b2)) {
            const uint32_t inst = __float_as_uint(a.w), prim = __float_as_uint(b.w);
            if ((__float_as_uint(c.w) & S2_TRI_ALPHA_TESTED) && !alpha(inst, prim, b1, b2)) continue;
            if (ANYHIT) {
                hit.t = t; hit.tri = ti; hit.instance = inst; hit.primitive = prim; hit.b1 = b1; hit.b2 = b2;
                return true;
            }
            // accepted hits have t <= hit.t; equal distances keep the lowest (instance, primitive)
            if (t < hit.t || inst < hit.instance || (inst == hit.instance && prim < hit.primitive)) {
                hit.t = t; hit.tri = ti; hit.instance = inst; hit.primitive = prim; hit.b1 = b1; hit.b2 = b2;
            }
        }
    }
    if (hits) {
        const uint32_t b = __ffs(hits) - 1;
        hits &= hits - 1;
        const uint32_t s = b ^ r.oct;
        const uint32_t next = child_base + __popc(imask & ((1u << s) - 1u));
        if (hits) {
            const uint2 g = make_uint2(child_base, imask | (hits << 8));
            if (st.sp < S2_STACK_SMEM) smem_stack[st.sp * lane_stride] = g;
            else if (st.sp < S2_STACK_DEPTH) lstack[st.sp - S2_STACK_SMEM] = g;
            else st.ok = false;
            if (st.sp < S2_STACK_DEPTH) st.sp++;
        }
        st.node = next;
        return false;
    }
    if (st.sp == 0) return true;
    // take the nearest remaining child of the top group; pop the group when it empties
    uint2 g = (st.sp - 1 < S2_STACK_SMEM) ? smem_stack[(st.sp - 1) * lane_stride] : lstack[st.sp - 1 - S2_STACK_SMEM];
    uint32_t gh = g.y >> 8;
    const uint32_t b = __ffs(gh) - 1;
    gh &= gh - 1;
    const uint32_t gi = g.y & 0xffu;
    const uint32_t s = b ^ r.oct;
    st.node = g.x + __popc(gi & ((1u << s) - 1u));
    if (gh) {
        g.y = gi | (gh << 8);
        if (st.sp - 1 < S2_STACK_SMEM) smem_stack[(st.sp - 1) * lane_stride] = g;
        else lstack[st.sp - 1 - S2_STACK_SMEM] = g;
    } else {
        st.sp--;
    }
    return false;
}

// Step of the warp-cooperative traversal with postponed triangle tests (the "while-while" order of
// Aila and Laine, HPG 2009, decided per step by a warp vote).  A lane alternates between node steps
// and triangle steps: a node step visits st.node, records the node's leaf triangles as pending
// (st.tbase, st.tmask) and moves to the next node; a lane with pending triangles takes no node step
// until they are tested, one per triangle step.  `do_tri` (warp-uniform) selects the step kind, so
// lanes in one step run the same code.  Returns true when the ray is finished (no node left and no
// triangle pending, or an accepted any-hit).
constexpr uint32_t kTravDone = 0xffffffffu;
// Tuning of the warp-cooperative traversal (runtime, chosen by s2_autotune): triangle tests per
// triangle step, and the vote: a triangle step when vote8 / 8 of the lanes with work have
// triangles pending (or no lane can take a node step).  Zero selects the defaults, measured on B200
// (terrain workload): 4 triangles, 4/8.
struct TravTuning {
    uint32_t tris_per_step;
    uint32_t vote8;
};

template <bool ANYHIT, bool COUNT, class Alpha = NoAlphaTest>
S2D bool trav_step_pp(const TravRay& r, TravState& st, const uint4* __restrict__ nodes4, const float4* __restrict__ tris4,
                      uint2* __restrict__ smem_stack, uint32_t lane_stride, uint2* lstack, TravHit& hit, TravCounters& ctr,
                      bool do_tri, uint32_t tris_per_step, const Alpha& alpha = Alpha()) {
    if (do_tri) {
        const uint32_t nt = tris_per_step ? tris_per_step : 4u;  // 0: the default
#pragma unroll 1
        for (uint32_t rep = 0; rep < nt && st.tmask; ++rep) {
            const uint32_t k = __ffs(st.tmask) - 1;
            st.tmask &= st.tmask - 1;
            const uint32_t ti = st.tbase + k;
            const float4 a = __ldg(tris4 + 3 * (size_t)ti + 0);
            const float4 b = __ldg(tris4 + 3 * (size_t)ti + 1);
            const float4 c = __ldg(tris4 + 3 * (size_t)ti + 2);
            if (COUNT) ctr.tris++;
            float t, b1, b2;
            if (intersect_triangle(r, ld3(a), ld3(b), ld3(c), hit.t, t, b1, b2)) {
                const uint32_t inst = __float_as_uint(a.w), prim = __float_as_uint(b.w);
                if (!((__float_as_uint(c.w) & S2_TRI_ALPHA_TESTED) && !alpha(inst, prim, b1, b2))) {
                    if (ANYHIT) {
                        hit.t = t; hit.tri = ti; hit.instance = inst; hit.primitive = prim; hit.b1 = b1; hit.b2 = b2;
                        st.tmask = 0;
                        st.node = kTravDone;
                        return true;
                    }
                    if (t < hit.t || inst < hit.instance || (inst == hit.instance && prim < hit.primitive)) {
                        hit.t = t; hit.tri = ti; hit.instance = inst; hit.primitive = prim; hit.b1 = b1; hit.b2 = b2;
                    }
                }
            }
        }
    } else if (st.tmask == 0 && st.node != kTravDone) {
        uint32_t child_base, imask, hits, tri_base, trimask;
        intersect_node(r, nodes4, st.node, hit.t, child_base, imask, hits, tri_base, trimask);
        if (COUNT) ctr.nodes++;
        st.tbase = tri_base;
        st.tmask = trimask;
        if (hits) {
            const uint32_t b = __ffs(hits) - 1;
            hits &= hits - 1;
            const uint32_t s = b ^ r.oct;
            const uint32_t next = child_base + __popc(imask & ((1u << s) - 1u));
            if (hits) {
                const uint2 g = make_uint2(child_base, imask | (hits << 8));
                if (st.sp < S2_STACK_SMEM) smem_stack[st.sp * lane_stride] = g;
                else if (st.sp < S2_STACK_DEPTH) lstack[st.sp - S2_STACK_SMEM] = g;
                else st.ok = false;
                if (st.sp < S2_STACK_DEPTH) st.sp++;
            }
            st.node = next;
        } else if (st.sp == 0) {
            st.node = kTravDone;
        } else {
            uint2 g = (st.sp - 1 < S2_STACK_SMEM) ? smem_stack[(st.sp - 1) * lane_stride] : lstack[st.sp - 1 - S2_STACK_SMEM];
            uint32_t gh = g.y >> 8;
            const uint32_t b = __ffs(gh) - 1;
            gh &= gh - 1;
            const uint32_t gi = g.y & 0xffu;
            const uint32_t s = b ^ r.oct;
            st.node = g.x + __popc(gi & ((1u << s) - 1u));
            if (gh) {
                g.y = gi | (gh << 8);
                if (st.sp - 1 < S2_STACK_SMEM) smem_stack[(st.sp - 1) * lane_stride] = g;
                else lstack[st.sp - 1 - S2_STACK_SMEM] = g;
            } else {
                st.sp--;
            }
        }
    }
    return st.tmask == 0 && st.node == kTravDone;
}

// Warp vote for trav_step_pp: a triangle step when at least vote8 / 8 of the lanes with work have
// triangles pending, or when no lane can take a node step.
S2D bool trav_vote_tri(bool active, const TravState& st, uint32_t vote8) {
    const uint32_t tri = __ballot_sync(0xffffffffu, active && st.tmask != 0);
    const uint32_t node = __ballot_sync(0xffffffffu, active && st.tmask == 0 && st.node != kTravDone);
    const uint32_t v = vote8 ? vote8 : 4u;  // 0: the default
    return node == 0u || 8u * (uint32_t)__popc(tri) >= v * (uint32_t)__popc(tri | node);
}

// Whole traversal of one ray.  ANYHIT: stop at the first accepted triangle.  COUNT: count node and
// triangle fetches into `ctr`.  Returns false if the stack overflowed (result may be incomplete).
template <bool ANYHIT, bool COUNT, class Alpha = NoAlphaTest>
S2D bool traverse(const TravRay& r, float tmax, const uint4* __restrict__ nodes4, const float4* __restrict__ tris4,
                  uint2* __restrict__ smem_stack, uint32_t lane_stride, TravHit& hit, TravCounters& ctr,
                  const Alpha& alpha = Alpha()) {
    uint2 lstack[S2_STACK_DEPTH - S2_STACK_SMEM];
    TravState st;
    trav_begin(st, hit, tmax);
    while (!trav_step<ANYHIT, COUNT, Alpha>(r, st, nodes4, tris4, smem_stack, lane_stride, lstack, hit, ctr, alpha)) {
    }
    return st.ok;
}
