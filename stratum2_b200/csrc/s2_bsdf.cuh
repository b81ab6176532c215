// BSDFs: Lambertian (src/Shaders/materials/lambertian.hlsli) and the Disney principled BSDF
// (src/Shaders/materials/disney.hlsli) with its microfacet helpers
// (src/Shaders/common/microfacet.hlsli), evaluated in the local shading frame.
#pragma once
#include "s2_shade.cuh"

// The shaders' pow(x, 5) as two squarings and a product (within a few ulp of powf, at a fraction of
// its instructions).
S2D float pow5(float x) { const float x2 = x * x; return x2 * x2 * x; }
// microfacet.hlsli:22-27
S2D float schlick1(float F0, float c) { return F0 + (1.f - F0) * pow5(fmaxf(1.f - c, 0.f)); }
S2D float3 schlick3(float3 F0, float c) { const float k = pow5(fmaxf(1.f - c, 0.f)); return F0 + (f3(1.f) - F0) * k; }
// microfacet.hlsli:42-62; IEEE-rounded division and square root (the reflectance ratios cancel
// near Brewster's angle, where an approximate quotient loses relative accuracy)
S2D float fresnel_dielectric(float ndi, float eta) {
    const float ndt2 = 1.f - __fdiv_rn(1.f - ndi * ndi, eta * eta);
    if (ndt2 < 0.f) return 1.f;
    const float ndt = __fsqrt_rn(ndt2), ni = fabsf(ndi);
    const float rs = __fdiv_rn(ni - eta * ndt, ni + eta * ndt), rp = __fdiv_rn(eta * ni - ndt, eta * ni + ndt);
    return (rs * rs + rp * rp) * 0.5f;
}
// microfacet.hlsli:64-81
S2D float gtr1(float ndh, float a) { const float a2 = a * a, t = 1.f + (a2 - 1.f) * ndh * ndh; return (a2 - 1.f) / (S2_PI * logf(a2) * t); }
S2D float gtr2(float3 h, float ax, float ay) {
    const float3 hs = f3(h.x / ax, h.y / ay, h.z);
    const float l2 = dot(hs, hs);
    return 1.f / (S2_PI * ax * ay * l2 * l2);
}
// microfacet.hlsli:101-111
S2D float smith_gtr2(float3 v, float ax, float ay) {
    const float lam = (-1.f + sqrtf(1.f + (v.x * v.x * ax * ax + v.y * v.y * ay * ay) / (v.z * v.z))) * 0.5f;
    return 1.f / (1.f + lam);
}
S2D float smith_gtr1(float3 v) { return smith_gtr2(v, 0.25f, 0.25f); }
// sample_visible_normals (microfacet.hlsli:148-179), Heitz 2018
S2D float3 sample_vndf(float3 in, float ax, float ay, float u1, float u2) {
    const bool flip = in.z < 0.f;
    if (flip) in = -in;
    const float3 hin = normalize(f3(ax * in.x, ay * in.y, in.z));
    const float r = sqrtf(u1), phi = 2.f * S2_PI * u2;
    const float t1 = r * cosf(phi);
    float t2 = r * sinf(phi);
    const float sc = (1.f + hin.z) * 0.5f;
    t2 = (1.f - sc) * sqrtf(1.f - t1 * t1) + sc * t2;
    const float3 disk = f3(t1, t2, sqrtf(fmaxf(0.f, 1.f - t1 * t1 - t2 * t2)));
    float3 f0, f1;
    make_orthonormal(hin, f0, f1);
    const float3 hN = f0 * disk.x + f1 * disk.y + hin * disk.z;
    const float3 out = normalize(f3(ax * hN.x, ay * hN.y, fmaxf(0.f, hN.z)));
    return flip ? -out : out;
}

template <class M>
S2D void disney_alphas(const M& m, float& ax, float& ay) {
    const float aspect = sqrtf(1.f - m.anisotropic() * 0.9f);
    const float a = pow2(m.roughness());
    ax = fmaxf(1e-4f, a / aspect);
    ay = fmaxf(1e-4f, a * aspect);
}

// Disney eval<Adjoint=false> (disney.hlsli:9-139): reflectance f*|cos|
template <class M>
S2D float3 disney_eval(const M& m, float3 in, float3 out) {
    float ax, ay;
    disney_alphas(m, ax, ay);
    const float metallic = m.metallic();
    if (in.z * out.z > 0.f) {
        const float ndi = fabsf(in.z), ndo = out.z;
        float3 h = normalize(in + out);
        if (h.z * in.z < 0.f) h = -h;
        const float ndh = h.z, hdi = dot(h, in), hdo = dot(h, out);
        float3 c = f3(0.f);
        if (in.z >= 0.f && out.z >= 0.f) {
            const float Fd90 = 0.5f + 2.f * m.roughness() * hdo * hdo;
            const float so = pow5(1.f - ndo), si = pow5(1.f - ndi), sh = pow5(1.f - hdo);
            const float base_diffuse = (1.f + (Fd90 - 1.f) * so) * (1.f + (Fd90 - 1.f) * si);
            const float Fss90 = hdo * hdo * m.roughness();
            const float Fss = (1.f + (Fss90 - 1.f) * so) * (1.f + (Fss90 - 1.f) * si);
            const float ss = 1.25f * (Fss * (1.f / (ndo + ndi) - 0.5f) + 0.5f);
            const float3 bc = m.base();
            c += bc * ((1.f - m.transmission()) * (1.f - metallic) * (lerpf(base_diffuse, ss, m.subsurface()) / S2_PI) * ndo);
            const float lb = luminance(bc);
            const float3 Ctint = lb > 0.f ? bc / lb : f3(1.f);
            const float3 Csheen = lerp3(f3(1.f), Ctint, 0.5f);
            c += Csheen * ((1.f - metallic) * m.sheen() * sh * ndo);
            if (ndi > 0.f && hdo > 0.f && ndh > 0.f) {
                const float eta = m.eta1();
                const float f0 = (eta - 1.f) * (eta - 1.f) / ((eta + 1.f) * (eta + 1.f));
                const float3 spec_color = lerp3(f3(1.f), Ctint, 0.5f);
                const float3 Cspec0 = lerp3(spec_color * (m.specular() * f0), bc, metallic);
                const float3 F = schlick3(Cspec0, hdo);
                const float D = gtr2(h, ax, ay), G = smith_gtr2(in, ax, ay) * smith_gtr2(out, ax, ay);
                const float sw = 1.f - m.transmission() * (1.f - metallic);
                c += F * (sw * D * G / (4.f * ndi));
            }
            if (ndi > 0.f && ndh > 0.f && m.clearcoat() > 0.f) {  // a zero clearcoat adds nothing
                const float ac = lerpf(0.1f, 0.001f, m.clearcoat_gloss());
                const float Fc = schlick1(0.04f, hdo), Dc = gtr1(ndh, ac), Gc = smith_gtr1(in) * smith_gtr1(out);
                c += f3(m.clearcoat() * Fc * Dc * Gc / (4.f * ndi));
            }
        }
        const float gw = (1.f - metallic) * m.transmission();
        if (gw > 0.f) {
            const float eta = in.z > 0.f ? m.eta1() : 1.f / m.eta1();
            const float Fg = fresnel_dielectric(hdi, eta), D = gtr2(h, ax, ay), G = smith_gtr2(in, ax, ay) * smith_gtr2(out, ax, ay);
            c += m.base() * (gw * (Fg * D * G) / (4.f * fabsf(ndi)));
        }
        return c;
    }
    const float gw = (1.f - metallic) * m.transmission();
    if (gw <= 0.f) return f3(0.f);
    const float eta = in.z > 0.f ? m.eta1() : 1.f / m.eta1();
    float3 h = normalize(in + out * eta);
    if (h.z * in.z < 0.f) h = -h;
    const float hdi = dot(h, in), hdo = dot(h, out), sd = hdi + eta * hdo;
    const float Fg = fresnel_dielectric(hdi, eta), D = gtr2(h, ax, ay), G = smith_gtr2(in, ax, ay) * smith_gtr2(out, ax, ay);
    return sqrt3(m.base()) * (gw * ((1.f - Fg) * D * G * eta * eta * fabsf(hdo * hdi)) / (fabsf(in.z) * sd * sd));
}

// Disney evalPdf (disney.hlsli:141-231)
template <class M>
S2D float disney_pdf(const M& m, float3 in, float3 out) {
    float ax, ay;
    disney_alphas(m, ax, ay);
    const float metallic = m.metallic(), tr = m.transmission();
    const float ac = (1.f - m.clearcoat_gloss()) * 0.1f + m.clearcoat_gloss() * 0.001f;
    const float dw = (1.f - metallic) * (1.f - tr), mw = 1.f - tr * (1.f - metallic), gw = (1.f - metallic) * tr, cw = m.clearcoat();
    const float tw = dw + mw + gw + cw;
    float dp = dw / tw, mp = mw / tw, gp = gw / tw, cp = cw / tw;
    if (in.z < 0.f) { dp = 0.f; mp = 0.f; cp = 0.f; if (gp > 0.f) gp = 1.f; }
    if (in.z * out.z > 0.f) {
        float3 h = normalize(in + out);
        if (h.z < 0.f) h = -h;
        const float ndi = in.z, ndh = h.z, hdi = dot(h, in), hdo = dot(h, out);
        if (in.z >= 0.f && out.z >= 0.f) {
            dp *= fmaxf(out.z, 0.f) / S2_PI;
            if (ndi > 0.f) mp *= gtr2(h, ax, ay) * smith_gtr2(in, ax, ay) / (4.f * ndi);
            else mp = 0.f;
            if (cp > 0.f) {  // lobes of zero weight skip their densities
                if (ndh > 0.f && hdo > 0.f) cp *= gtr1(ndh, ac) * ndh / (4.f * hdo);
                else cp = 0.f;
            }
        }
        if (gp > 0.f) {
            const float eta = in.z > 0.f ? m.eta1() : 1.f / m.eta1();
            gp *= fresnel_dielectric(hdi, eta) * gtr2(h, ax, ay) * smith_gtr2(in, ax, ay) / (4.f * fabsf(ndi));
        }
    } else if (gp > 0.f) {
        const float eta = in.z > 0.f ? m.eta1() : 1.f / m.eta1();
        float3 h = normalize(in + out * eta);
        if (h.z < 0.f) h = -h;
        const float hdi = dot(h, in), hdo = dot(h, out);
        const float D = gtr2(h, ax, ay), Gi = smith_gtr2(in, ax, ay), Fg = fresnel_dielectric(hdi, eta);
        const float sd = hdi + eta * hdo, dh = eta * eta * hdo / (sd * sd);
        gp *= (1.f - Fg) * D * Gi * fabsf(dh * hdi / in.z);
    }
    return dp + mp + gp + cp;
}

// Disney sample (disney.hlsli:233-380).  Returns false on a failed sample (zero direction);
// rough = 0 marks a singular sample.
template <class M>
S2D bool disney_sample(const M& m, float3 in, float r0, float r1, float r2, float3& dir, float& rough) {
    float ax, ay;
    disney_alphas(m, ax, ay);
    const float ac = (1.f - m.clearcoat_gloss()) * 0.1f + m.clearcoat_gloss() * 0.001f;
    const float metallic = m.metallic(), tr = m.transmission();
    const float dw = (1.f - metallic) * (1.f - tr), mw = 1.f - tr * (1.f - metallic), gw = (1.f - metallic) * tr, cw = m.clearcoat();
    if (in.z >= 0.f) {
        const float tw = dw + mw + gw + cw;
        const float dp = dw / tw, mp = mw / tw, gp = gw / tw;
        if (r2 <= dp) { dir = sample_cos_hemisphere(r0, r1); rough = 1.f; return true; }
        if (r2 <= dp + mp) {
            const float3 h = sample_vndf(in, ax, ay, r0, r1);
            dir = normalize(-in + h * (2.f * dot(in, h)));
            rough = m.roughness();
            return true;
        }
        if (r2 <= dp + mp + gp) {
            if (gp <= 0.f) { dir = f3(0.f); rough = 0.f; return false; }
            float3 h = sample_vndf(in, ax, ay, r0, r1);
            const float hdi = dot(h, in), eta = in.z > 0.f ? m.eta1() : 1.f / m.eta1();
            const float F = fresnel_dielectric(hdi, eta), u = (r2 - (dp + mp)) / gp;
            if (u <= F) { dir = normalize(-in + h * (2.f * dot(in, h))); rough = 0.f; return true; }
            const float hdo2 = 1.f - (1.f - hdi * hdi) / (eta * eta);
            if (hdo2 <= 0.f) { dir = f3(0.f); rough = 0.f; return false; }
            if (hdi < 0.f) h = -h;
            dir = -in / eta + h * (fabsf(hdi) / eta - sqrtf(hdo2));
            rough = m.roughness();
            return true;
        }
        const float a2 = ac * ac;
        const float ch = sqrtf(fmaxf(0.f, (1.f - powf(a2, 1.f - r0)) / (1.f - a2)));
        const float sh = sqrtf(fmaxf(1.f - ch * ch, 0.f)), az = 2.f * S2_PI * r1;
        const float3 mn = f3(sh * cosf(az), sh * sinf(az), ch);
        dir = normalize(-in + mn * (2.f * dot(in, mn)));
        rough = sqrtf(ac);
        return true;
    }
    float3 h = sample_vndf(in, ax, ay, r0, r1);
    if (h.z < 0.f) h = -h;
    const float hdi = dot(h, in), eta = in.z > 0.f ? m.eta1() : 1.f / m.eta1();
    const float F = fresnel_dielectric(hdi, eta);
    if (r2 <= F) { dir = normalize(-in + h * (2.f * dot(in, h))); rough = m.roughness(); return true; }
    const float hdo2 = 1.f - (1.f - hdi * hdi) / (eta * eta);
    if (hdo2 <= 0.f) { dir = f3(0.f); rough = 0.f; return false; }
    if (hdi < 0.f) h = -h;
    dir = -in / eta + h * (fabsf(hdi) / eta - sqrtf(hdo2));
    rough = m.roughness();
    return true;
}

// evaluateReflectance: f*|cos|, forward and reverse pdf (lambertian.hlsli:16-27, disney.hlsli:391-403)
template <bool LAMBERT, class M>
S2D void bsdf_eval(const M& m, float3 in, float3 out, float3& f, float& fwd, float& rev) {
    if (LAMBERT) {
        if (in.z * out.z < 0.f) { f = f3(0.f); fwd = rev = 0.f; return; }
        f = m.base() * (fabsf(out.z) / S2_PI);
        fwd = cos_hemisphere_pdfw(fmaxf(1e-5f, fabsf(out.z)));
        rev = cos_hemisphere_pdfw(fmaxf(1e-5f, fabsf(in.z)));
        return;
    }
    f = disney_eval(m, in, out);
    fwd = disney_pdf(m, in, out);
    rev = disney_pdf(m, out, in);
}

// sampleDirection (lambertian.hlsli:29-38, disney.hlsli:415-429)
template <bool LAMBERT, class M>
S2D void bsdf_sample(const M& m, float3 in, float4 rnd, float3& dir, float3& f, float& fwd, float& rev, float& rough) {
    if (LAMBERT) {
        dir = sample_cos_hemisphere(rnd.x, rnd.y);
        if (in.z < 0.f) dir = -dir;
        f = m.base() * (fabsf(dir.z) / S2_PI);
        fwd = cos_hemisphere_pdfw(fmaxf(1e-5f, fabsf(dir.z)));
        rev = cos_hemisphere_pdfw(fmaxf(1e-5f, fabsf(in.z)));
        rough = 1.f;
        return;
    }
    disney_sample(m, in, rnd.x, rnd.y, rnd.z, dir, rough);
    bsdf_eval<false>(m, in, dir, f, fwd, rev);
}

template <bool LAMBERT, class M>
S2D bool mat_singular(const M& m) {
    if (LAMBERT) return false;
    // disney.hlsli:387
    return fmaxf(fmaxf(m.specular(), m.metallic()), m.transmission()) * (1.f - m.roughness()) > 0.75f;
}
template <class M>
S2D float cont_prob(const M& m) { return saturate(luminance(m.base())); }
