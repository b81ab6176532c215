// ORACLE -- test infrastructure only (included by oracle/oracle.cpp).
// Restatement of the camera-path tracer of src/Shaders/kernels/testrenderer.slang (TestRenderer,
// gMultiDispatch + gDeferShadowRays + gSampleDirectIllumination defaults, TestRenderer.cpp:19-36)
// with the minPathLength gate of src/Shaders/kernels/vcm.slang:922,960,977.
//
// Deliberate differences from the reference shaders (each is a defect there):
//  * environment NEE uses the sampled direction; the reference leaves
//    IlluminationSampleRecord.mDirectionToLight unset for environment samples (lights.hlsli:234-244);
//  * the MIS weight of a BSDF-sampled environment hit uses the environment's solid-angle pdf; the
//    reference passes the light-tracing disc pdf 1/(pi R^2) (testrenderer.slang:1047-1050) unless
//    S2_FLAG_REFERENCE_ENV_MIS is set;
//  * after a vertex whose material is singular (NEE skipped, testrenderer.slang:869) the next
//    emission hit gets weight 1; the reference still MIS-weights it (:905-913);
//  * a half-precision pdf that overflows to infinity gives MIS weight 1 instead of NaN.
// NEE contributions accumulate in floating point instead of 1/16384 fixed point (:237-244).
namespace orc {

constexpr uint32_t FLAG_PIXEL_JITTER = 1u << 0, FLAG_LAMBERTIAN = 1u << 1, FLAG_PCG32 = 1u << 2, FLAG_NO_NEE = 1u << 3,
                   FLAG_RESTIR = 1u << 4, FLAG_REF_ENV_MIS = 1u << 5, FLAG_NO_RR = 1u << 6, FLAG_NO_SHADING_NORMALS = 1u << 8,
                   FLAG_RESTIR_REUSE = 1u << 11, FLAG_NO_ALPHA = 1u << 12,
                   FLAG_NO_NORMAL_MAPS = 1u << 13, FLAG_RESTIR_REUSE_VIS = 1u << 18,
                   FLAG_F32_MATERIALS = 1u << 30;  // oracle only: the materials of s2_render_diff

template <class R> R un8(uint32_t w, int shift) { return R((w >> shift) & 0xffu) / R(255); }
inline uint32_t pk8(double v) { v = std::min(std::max(v, 0.0), 1.0); return (uint32_t)std::floor((float)v * 255.f + 0.5f); }

// PackedMaterialData (compat/material_data.h:12-73)
// With `f32` set (the differentiable renderer's materials) the getters return the unquantised
// parameters in `f` instead: base rgb, emission rgb, then specular .. eta as in the packed order.
template <class R> struct Mat {
    uint32_t w[4];
    R escale;
    bool f32 = false;
    R f[16];
    V3<R> base() const { return f32 ? V3<R>(f[0], f[1], f[2]) : V3<R>(un8<R>(w[0], 0), un8<R>(w[0], 8), un8<R>(w[0], 16)); }
    V3<R> emission() const {
        return f32 ? V3<R>(f[3], f[4], f[5]) : V3<R>(un8<R>(w[1], 0), un8<R>(w[1], 8), un8<R>(w[1], 16)) * escale;
    }
    R specular() const { return f32 ? f[6] : un8<R>(w[0], 24); }
    R sheen() const { return f32 ? f[7] : un8<R>(w[1], 24); }
    R metallic() const { return f32 ? f[8] : un8<R>(w[2], 0); }
    R roughness() const { return f32 ? f[9] : un8<R>(w[2], 8); }
    R anisotropic() const { return f32 ? f[10] : un8<R>(w[2], 16); }
    R subsurface() const { return f32 ? f[11] : un8<R>(w[2], 24); }
    R clearcoat() const { return f32 ? f[12] : un8<R>(w[3], 0); }
    R clearcoat_gloss() const { return f32 ? f[13] : un8<R>(w[3], 8); }
    R transmission() const { return f32 ? f[14] : un8<R>(w[3], 16); }
    R eta1() const { return (f32 ? f[15] : un8<R>(w[3], 24)) + 1; }
    void set_base(const V3<R>& c) {
        w[0] = (w[0] & 0xff000000u) | pk8(c.x) | pk8(c.y) << 8 | pk8(c.z) << 16;
    }
    void set_emission(V3<R> c) {
        escale = std::max(std::max(c.x, c.y), c.z);
        c = c / escale;
        auto q = [](R v) { return std::isnan(v) ? 0u : pk8(v); };
        w[1] = (w[1] & 0xff000000u) | q(c.x) | q(c.y) << 8 | q(c.z) << 16;
    }
};

template <class R> struct SD {
    V3<R> pos;
    uint32_t mat;
    uint32_t ng, ns, tg;
    R area;
    R u, v;
    V3<R> n, t, b, gn;  // unpacked frame
    bool surface() const { return area > 0; }
    void unpack() {
        n = unpack_normal<R>(ns); t = unpack_normal<R>(tg); b = cross(n, t); gn = unpack_normal<R>(ng);
    }
    V3<R> to_local(const V3<R>& v) const { return V3<R>(dot(v, t), dot(v, b), dot(v, n)); }
    V3<R> to_world(const V3<R>& v) const { return t * v.x + b * v.y + n * v.z; }
    // shadingNormalCorrection<false> (shading_data.hlsli:35-55)
    R snc(const V3<R>& in, const V3<R>& out) const {
        const V3<R> lg = to_local(gn);
        const R a = dot(lg, in), c = dot(lg, out);
        auto sg = [](R x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); };
        if (sg(c) != sg(out.z) || sg(a) != sg(in.z)) return 0;
        return 1;
    }
};

struct Params {
    uint32_t min_len, max_len, spp, seed, flags, restir_m;
    float exposure, env_prob;
    float max_m = 3.f;
};

// pcg / xxhash32 (rng.hlsli:5-22): the hash-grid keys
inline uint32_t pcg_hash(uint32_t v) {
    const uint32_t state = v * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
inline uint32_t xxhash32(uint32_t p) {
    uint32_t h = p + 374761393u;
    h = 668265263u * ((h << 17) | (h >> 15));
    h = 2246822519u * (h ^ (h >> 15));
    h = 3266489917u * (h ^ (h >> 13));
    return h ^ (h >> 16);
}

// HashGridData of the ReSTIR DI reuse (testrenderer.slang:152-168)
template <class R> struct GridRecord {
    V3<R> local_pos;
    uint32_t inst = 0, prim = 0;
    float rnd[4] = {0, 0, 0, 0};
    R target = 0, W = 0, M = 0;
    V3<R> dir_in;
};

// HashGrid<T> (hashgrid.hlsli:14-119) and GpuHashGrid::clear/build (GpuHashGrid.cpp:71-111),
// sequential: appends are serialised by a mutex and the per-cell offsets are a prefix sum in
// cell order (the GPU assigns them in atomic order; only the order inside a cell differs).
template <class R> struct CpuGrid {
    uint32_t cells = 0, max_size = 0;
    float min_cell = 0.5f, pixel_radius = 0.f, dscale = 0.f;
    V3<R> cam;
    std::vector<uint32_t> checksum, counter, offset, data_index;
    std::vector<GridRecord<R>> data;
    std::vector<std::pair<uint32_t, uint32_t>> app;
    std::mutex mu;

    void clear(uint32_t c, uint32_t size) {
        cells = c; max_size = size;
        checksum.assign(c, 0u); counter.assign(c, 0u); offset.assign(c, 0u);
        data.clear(); app.clear(); data_index.clear();
    }
    // GetCellSize (hashgrid.hlsli:43-49)
    float cell_size(const V3<R>& pos) const {
        if (pixel_radius <= 0.f) return min_cell;
        const float step = (float)length(cam - pos) * dscale;
        const float l = std::log2(step / min_cell);
        const uint32_t e = l > 0.f ? std::min<uint32_t>((uint32_t)l, 31u) : 0u;
        return min_cell * (float)(1u << e);
    }
    // FindCellIndex (hashgrid.hlsli:51-75)
    uint32_t find(const V3<R>& pos, float cs, bool insert) {
        const int x = (int)std::floor((float)pos.x / cs), y = (int)std::floor((float)pos.y / cs), z = (int)std::floor((float)pos.z / cs);
        uint32_t cb; std::memcpy(&cb, &cs, 4);
        const uint32_t sum = std::max(1u, xxhash32(xxhash32(cb) + xxhash32((uint32_t)z + xxhash32((uint32_t)y + xxhash32((uint32_t)x)))));
        const uint32_t base = pcg_hash(pcg_hash(cb) + pcg_hash((uint32_t)z + pcg_hash((uint32_t)y + pcg_hash((uint32_t)x)))) % cells;
        for (uint32_t i = 0; i < 32; ++i) {
            const uint32_t c = (base + i) % cells;
            if (insert && checksum[c] == 0u) { checksum[c] = sum; return c; }
            if (checksum[c] == sum) return c;
        }
        return 0xffffffffu;
    }
    // Append (hashgrid.hlsli:77-97)
    void append(const V3<R>& pos, const GridRecord<R>& rec) {
        std::lock_guard<std::mutex> lk(mu);
        const uint32_t c = find(pos, cell_size(pos), true);
        if (c == 0xffffffffu || data.size() >= max_size) return;
        app.emplace_back(c, counter[c]++);
        data.push_back(rec);
    }
    // ComputeIndices + Swizzle (hashgrid.hlsli:101-119)
    void build() {
        uint32_t acc = 0;
        for (uint32_t c = 0; c < cells; ++c) { offset[c] = acc; acc += counter[c]; }
        data_index.assign(data.size(), 0u);
        for (uint32_t i = 0; i < (uint32_t)data.size(); ++i) data_index[offset[app[i].first] + app[i].second] = i;
    }
};

template <class R> struct Tracer {
    const Scene<R>& s;
    Params p;
    uint64_t ext_rays = 0, shadow_rays = 0;
    CpuGrid<R>* grid_cur = nullptr;    // ReSTIR DI reuse: grid appended to by this call
    CpuGrid<R>* grid_prev = nullptr;   // the previous call's grid (null: none)
    // Detached sampling (test infrastructure for the adjoint renderer): materials for sampling
    // decisions, pdfs, MIS and Russian roulette come from this scene (same geometry, other images),
    // BSDF values and emission from `s`; null: both from `s`.
    const Scene<R>* samp = nullptr;
    Tracer(const Scene<R>& sc, const Params& pp) : s(sc), p(pp) {}

    bool has_env() const { return s.env_addr != S2_NO_ENVIRONMENT; }
    uint32_t light_count() const { return (uint32_t)s.light_map.size(); }

    // makeTriangleShadingData (shading_data.hlsli:59-151)
    SD<R> shading(uint32_t inst, uint32_t prim, R b1, R b2) const {
        SD<R> r;
        r.mat = (s.inst_word0[inst] >> 4);
        const R* M = &s.xf[12 * (size_t)inst];
        uint32_t idx[3]; s.tri_indices(inst, prim, idx);
        const V3<R> v0 = s.position(inst, idx[0]), v1 = s.position(inst, idx[1]), v2 = s.position(inst, idx[2]);
        const V3<R> dPds = s.xvec(M, v0 - v2), dPdt = s.xvec(M, v1 - v2);
        V3<R> gn = cross(dPds, dPdt);
        const R area2 = length(gn);
        gn = gn / area2;
        r.ng = pack_normal(gn);
        r.area = area2 / 2;
        R t0[2] = {0, 0}, t1[2] = {0, 0}, t2[2] = {0, 0};
        if (s.attr2(inst, idx[0], t0)) { s.attr2(inst, idx[1], t1); s.attr2(inst, idx[2], t2); }
        const R duvds[2] = {t2[0] - t0[0], t2[1] - t0[1]}, duvdt[2] = {t2[0] - t1[0], t2[1] - t1[1]};
        r.u = t0[0] + (t1[0] - t0[0]) * b1 + duvds[0] * b2;
        r.v = t0[1] + (t1[1] - t0[1]) * b1 + duvds[1] * b2;
        const R det = duvds[0] * duvdt[1] - duvdt[0] * duvds[1];
        V3<R> dPdu;
        R dsdu = 0, dtdu = 0, dsdv = 0, dtdv = 0;
        if (det != 0) {
            const R id = R(1) / det;
            dsdu = duvdt[1] * id; dtdu = -duvds[1] * id; dsdv = duvdt[0] * id; dtdv = -duvds[0] * id;
            dPdu = -(dPds * dsdu + dPdt * dtdu);
        } else {
            V3<R> tt, bb; make_orthonormal(gn, tt, bb); dPdu = tt;
        }
        bool valid = false;
        V3<R> sn, n0, n1, n2;
        if (!(p.flags & FLAG_NO_SHADING_NORMALS) && s.attr_normal(inst, idx[0], n0)) {
            s.attr_normal(inst, idx[1], n1); s.attr_normal(inst, idx[2], n2);
            sn = n0 + (n1 - n0) * b1 + (n2 - n0) * b2;
            valid = !((sn.x == 0 && sn.y == 0 && sn.z == 0) || std::isnan(sn.x) || std::isnan(sn.y) || std::isnan(sn.z));
        }
        if (!valid) {
            r.ns = r.ng;
            r.tg = pack_normal(normalize(dPdu));
        } else {
            sn = normalize(s.xvec(M, sn));
            const V3<R> tangent = normalize(dPdu - sn * dot(sn, dPdu));
            r.ns = pack_normal(sn);
            r.tg = pack_normal(tangent);
            if (dot(sn, gn) < 0) r.ng = pack_normal(-gn);
        }
        r.pos = s.xpoint(M, v0 + (v1 - v0) * b1 + (v2 - v0) * b2);
        r.unpack();
        return r;
    }

    V3<R> sample_image(uint32_t img, R u, R v) const { return s.images[img].sample(u, v); }

    // ApplyNormalMap (material.hlsli:78-105): bump image index, strength and channel count at
    // bytes 36..47 of the material record; bitangent sign +1
    void normal_map(SD<R>& sd) const {
        const uint32_t img = s.u32(s.mat, sd.mat + 36), channels = s.u32(s.mat, sd.mat + 44);
        const R scale = (R)s.f32(s.mat, sd.mat + 40);
        if (img >= s.images.size() || !(scale > 0)) return;
        R a;
        const V3<R> t = s.images[img].sample(sd.u, sd.v, &a);
        V3<R> bump = channels == 2 ? V3<R>(t.x, t.y, 1) : t;
        bump.x = (bump.x * 2 - 1) * scale;
        bump.y = -(bump.y * 2 - 1) * scale;
        const V3<R> n = normalize(sd.t * bump.x + cross(sd.n, sd.t) * bump.y + sd.n * bump.z);
        const V3<R> tg = normalize(sd.t - n * dot(n, sd.t));
        sd.ns = pack_normal(n);
        sd.tg = pack_normal(tg);
        sd.unpack();
    }

    // makeTriangleShadingData from an object-space position (shading_data.hlsli:153-173)
    SD<R> shading_local(uint32_t inst, uint32_t prim, const V3<R>& lp) const {
        uint32_t idx[3]; s.tri_indices(inst, prim, idx);
        const V3<R> v0 = s.position(inst, idx[0]), v1 = s.position(inst, idx[1]), v2 = s.position(inst, idx[2]);
        const V3<R> e1 = v1 - v0, e2 = v2 - v0, pv = lp - v0;
        const R d00 = dot(e1, e1), d01 = dot(e1, e2), d11 = dot(e2, e2), d20 = dot(pv, e1), d21 = dot(pv, e2);
        const R den = d00 * d11 - d01 * d01;
        SD<R> r = shading(inst, prim, (d11 * d20 - d01 * d21) / den, (d00 * d21 - d01 * d20) / den);
        r.pos = s.xpoint(&s.xf[12 * (size_t)inst], lp);
        return r;
    }

    // LoadMaterial (material.hlsli:15-46)
    Mat<R> material(uint32_t addr, R u, R v, const Scene<R>* sc = nullptr) const {
        const Scene<R>& S = sc ? *sc : s;
        Mat<R> m;
        for (int k = 0; k < 4; ++k) m.w[k] = S.u32(S.mat, addr + 4 * k);
        uint32_t img[4];
        for (int k = 0; k < 4; ++k) img[k] = S.u32(S.mat, addr + 16 + 4 * k);
        m.escale = (R)S.f32(S.mat, addr + 32);
        const uint32_t nimg = (uint32_t)S.images.size();
        if (p.flags & FLAG_F32_MATERIALS) {
            // the differentiable renderer's materials: texture modulation in floating point
            const V3<R> b = m.base(), e = m.emission();
            const R q[16] = {b.x, b.y, b.z, e.x, e.y, e.z, m.specular(), m.sheen(), m.metallic(), m.roughness(),
                             m.anisotropic(), m.subsurface(), m.clearcoat(), m.clearcoat_gloss(), m.transmission(),
                             un8<R>(m.w[3], 24)};
            for (int k = 0; k < 16; ++k) m.f[k] = q[k];
            m.f32 = true;
            if (img[0] < nimg) { const V3<R> t = S.images[img[0]].sample(u, v); m.f[0] *= t.x; m.f[1] *= t.y; m.f[2] *= t.z; }
            if (img[1] < nimg) { const V3<R> t = S.images[img[1]].sample(u, v); m.f[3] *= t.x; m.f[4] *= t.y; m.f[5] *= t.z; }
            if (img[2] < nimg) {
                R a; const V3<R> t = S.images[img[2]].sample(u, v, &a);
                m.f[8] *= t.x; m.f[9] = 1 - (1 - m.f[9]) * (1 - t.y); m.f[10] *= t.z; m.f[11] *= a;
            }
            if (img[3] < nimg) {
                R a; const V3<R> t = S.images[img[3]].sample(u, v, &a);
                m.f[12] *= t.x; m.f[13] *= t.y; m.f[14] *= t.z; m.f[15] *= a;
            }
            return m;
        }
        if (img[0] < nimg) m.set_base(m.base() * S.images[img[0]].sample(u, v));
        if (img[1] < nimg) m.set_emission(m.emission() * S.images[img[1]].sample(u, v));
        if (img[2] < nimg) {
            R a; const V3<R> vi = S.images[img[2]].sample(u, v, &a);
            R x = un8<R>(m.w[2], 0) * vi.x, y = 1 - (1 - un8<R>(m.w[2], 8)) * (1 - vi.y), z = un8<R>(m.w[2], 16) * vi.z, ww = un8<R>(m.w[2], 24) * a;
            m.w[2] = pk8(x) | pk8(y) << 8 | pk8(z) << 16 | pk8(ww) << 24;
        }
        if (img[3] < nimg) {
            R a; const V3<R> vi = S.images[img[3]].sample(u, v, &a);
            m.w[3] = pk8(un8<R>(m.w[3], 0) * vi.x) | pk8(un8<R>(m.w[3], 8) * vi.y) << 8 | pk8(un8<R>(m.w[3], 16) * vi.z) << 16 | pk8(un8<R>(m.w[3], 24) * a) << 24;
        }
        return m;
    }

    // ---------------------------------------------------------------- BSDFs
    bool lambert() const { return (p.flags & FLAG_LAMBERTIAN) != 0; }
    bool can_eval(const Mat<R>& m) const { return any_pos(m.base()); }
    bool singular(const Mat<R>& m) const {
        if (lambert()) return false;
        return std::max(std::max(m.specular(), m.metallic()), m.transmission()) * (1 - m.roughness()) > R(0.75);
    }
    R cont_prob(const Mat<R>& m) const { return sat(luminance(m.base())); }

    // microfacet.hlsli
    static R schlick(R F0, R c) { return F0 + (1 - F0) * std::pow(std::max(1 - c, R(0)), R(5)); }
    static V3<R> schlick3(const V3<R>& F0, R c) { const R k = std::pow(std::max(1 - c, R(0)), R(5)); return F0 + (V3<R>(1) - F0) * k; }
    static R fresnel_dielectric(R ndi, R eta) {
        const R ndt2 = 1 - (1 - ndi * ndi) / (eta * eta);
        if (ndt2 < 0) return 1;
        const R ndt = std::sqrt(ndt2), ni = std::fabs(ndi);
        const R rs = (ni - eta * ndt) / (ni + eta * ndt), rp = (eta * ni - ndt) / (eta * ni + ndt);
        return (rs * rs + rp * rp) / 2;
    }
    static R GTR1(R ndh, R a) { const R a2 = a * a, t = 1 + (a2 - 1) * ndh * ndh; return (a2 - 1) / (PI<R>() * std::log(a2) * t); }
    static R GTR2(const V3<R>& h, R ax, R ay) {
        const V3<R> hs(h.x / ax, h.y / ay, h.z);
        const R l2 = dot(hs, hs);
        return 1 / (PI<R>() * ax * ay * l2 * l2);
    }
    static R smith_gtr2(const V3<R>& v, R ax, R ay) {
        const R lam = (-1 + std::sqrt(1 + (v.x * v.x * ax * ax + v.y * v.y * ay * ay) / (v.z * v.z))) / 2;
        return 1 / (1 + lam);
    }
    static R smith_gtr1(const V3<R>& v) { return smith_gtr2(v, R(0.25), R(0.25)); }
    static V3<R> sample_vndf(V3<R> in, R ax, R ay, R u1, R u2) {
        const bool flip = in.z < 0;
        if (flip) in = -in;
        const V3<R> hin = normalize(V3<R>(ax * in.x, ay * in.y, in.z));
        const R r = std::sqrt(u1), phi = 2 * PI<R>() * u2;
        const R t1 = r * std::cos(phi);
        R t2 = r * std::sin(phi);
        const R sc = (1 + hin.z) / 2;
        t2 = (1 - sc) * std::sqrt(1 - t1 * t1) + sc * t2;
        const V3<R> disk(t1, t2, std::sqrt(std::max(R(0), 1 - t1 * t1 - t2 * t2)));
        V3<R> f0, f1; make_orthonormal(hin, f0, f1);
        const V3<R> hN = f0 * disk.x + f1 * disk.y + hin * disk.z;
        V3<R> out = normalize(V3<R>(ax * hN.x, ay * hN.y, std::max(R(0), hN.z)));
        return flip ? -out : out;
    }

    void alphas(const Mat<R>& m, R& ax, R& ay) const {
        const R aspect = std::sqrt(1 - m.anisotropic() * R(0.9));
        const R a = pow2(m.roughness());
        ax = std::max(R(1e-4), a / aspect); ay = std::max(R(1e-4), a * aspect);
    }

    // Disney eval (disney.hlsli:9-139), Adjoint = false
    V3<R> disney_eval(const Mat<R>& m, const V3<R>& in, const V3<R>& out) const {
        R ax, ay; alphas(m, ax, ay);
        const R metallic = m.metallic();
        if (in.z * out.z > 0) {
            const R ndi = std::fabs(in.z), ndo = out.z;
            V3<R> h = normalize(in + out);
            if (h.z * in.z < 0) h = -h;
            const R ndh = h.z, hdi = dot(h, in), hdo = dot(h, out);
            V3<R> c(0);
            if (in.z >= 0 && out.z >= 0) {
                const R Fd90 = R(0.5) + 2 * m.roughness() * hdo * hdo;
                const R so = std::pow(1 - ndo, R(5)), si = std::pow(1 - ndi, R(5)), sh = std::pow(1 - hdo, R(5));
                const R base_diffuse = (1 + (Fd90 - 1) * so) * (1 + (Fd90 - 1) * si);
                const R Fss90 = hdo * hdo * m.roughness();
                const R Fss = (1 + (Fss90 - 1) * so) * (1 + (Fss90 - 1) * si);
                const R ss = R(1.25) * (Fss * (1 / (ndo + ndi) - R(0.5)) + R(0.5));
                const V3<R> bc = m.base();
                c = c + bc * ((1 - m.transmission()) * (1 - metallic) * (lerp1(base_diffuse, ss, m.subsurface()) / PI<R>()) * ndo);
                const R lb = luminance(bc);
                const V3<R> Ctint = lb > 0 ? bc / lb : V3<R>(1);
                const V3<R> Csheen = lerp3(V3<R>(1), Ctint, R(0.5));
                c = c + Csheen * ((1 - metallic) * m.sheen() * sh * ndo);
                if (ndi > 0 && hdo > 0 && ndh > 0) {
                    const R eta = m.eta1();
                    const R f0 = (eta - 1) * (eta - 1) / ((eta + 1) * (eta + 1));
                    const V3<R> spec_color = lerp3(V3<R>(1), Ctint, R(0.5));
                    const V3<R> Cspec0 = lerp3(spec_color * (m.specular() * f0), bc, metallic);
                    const V3<R> F = schlick3(Cspec0, hdo);
                    const R D = GTR2(h, ax, ay), G = smith_gtr2(in, ax, ay) * smith_gtr2(out, ax, ay);
                    const R sw = 1 - m.transmission() * (1 - metallic);
                    c = c + F * (sw * D * G / (4 * ndi));
                }
                if (ndi > 0 && ndh > 0) {
                    const R ac = lerp1(R(0.1), R(0.001), m.clearcoat_gloss());
                    const R Fc = schlick(R(0.04), hdo), Dc = GTR1(ndh, ac), Gc = smith_gtr1(in) * smith_gtr1(out);
                    c = c + V3<R>(m.clearcoat() * Fc * Dc * Gc / (4 * ndi));
                }
            }
            const R gw = (1 - metallic) * m.transmission();
            if (gw > 0) {
                const R eta = in.z > 0 ? m.eta1() : 1 / m.eta1();
                const R Fg = fresnel_dielectric(hdi, eta), D = GTR2(h, ax, ay), G = smith_gtr2(in, ax, ay) * smith_gtr2(out, ax, ay);
                c = c + m.base() * (gw * (Fg * D * G) / (4 * std::fabs(ndi)));
            }
            return c;
        }
        const R gw = (1 - metallic) * m.transmission();
        if (gw <= 0) return V3<R>(0);
        const R eta = in.z > 0 ? m.eta1() : 1 / m.eta1();
        V3<R> h = normalize(in + out * eta);
        if (h.z * in.z < 0) h = -h;
        const R hdi = dot(h, in), hdo = dot(h, out), sd = hdi + eta * hdo;
        const R Fg = fresnel_dielectric(hdi, eta), D = GTR2(h, ax, ay), G = smith_gtr2(in, ax, ay) * smith_gtr2(out, ax, ay);
        const V3<R> bc = m.base();
        return V3<R>(std::sqrt(bc.x), std::sqrt(bc.y), std::sqrt(bc.z)) *
               (gw * ((1 - Fg) * D * G * eta * eta * std::fabs(hdo * hdi)) / (std::fabs(in.z) * sd * sd));
    }

    // Disney evalPdf (disney.hlsli:141-231)
    R disney_pdf(const Mat<R>& m, const V3<R>& in, const V3<R>& out) const {
        R ax, ay; alphas(m, ax, ay);
        const R metallic = m.metallic();
        const R ac = (1 - m.clearcoat_gloss()) * R(0.1) + m.clearcoat_gloss() * R(0.001);
        const R tr = m.transmission();
        const R dw = (1 - metallic) * (1 - tr), mw = (1 - tr * (1 - metallic)), gw = (1 - metallic) * tr, cw = m.clearcoat();
        const R tw = dw + mw + gw + cw;
        R dp = dw / tw, mp = mw / tw, gp = gw / tw, cp = cw / tw;
        if (in.z < 0) { dp = 0; mp = 0; cp = 0; if (gp > 0) gp = 1; }
        if (in.z * out.z > 0) {
            V3<R> h = normalize(in + out);
            if (h.z < 0) h = -h;
            const R ndi = in.z, ndh = h.z, hdi = dot(h, in), hdo = dot(h, out);
            if (in.z >= 0 && out.z >= 0) {
                dp *= std::max(out.z, R(0)) / PI<R>();
                if (ndi > 0) mp *= GTR2(h, ax, ay) * smith_gtr2(in, ax, ay) / (4 * ndi);
                else mp = 0;
                if (ndh > 0 && hdo > 0) cp *= GTR1(ndh, ac) * ndh / (4 * hdo);
                else cp = 0;
            }
            const R eta = in.z > 0 ? m.eta1() : 1 / m.eta1();
            gp *= fresnel_dielectric(hdi, eta) * GTR2(h, ax, ay) * smith_gtr2(in, ax, ay) / (4 * std::fabs(ndi));
        } else {
            const R eta = in.z > 0 ? m.eta1() : 1 / m.eta1();
            V3<R> h = normalize(in + out * eta);
            if (h.z < 0) h = -h;
            const R hdi = dot(h, in), hdo = dot(h, out);
            const R D = GTR2(h, ax, ay), Gi = smith_gtr2(in, ax, ay), Fg = fresnel_dielectric(hdi, eta);
            const R sd = hdi + eta * hdo, dh = eta * eta * hdo / (sd * sd);
            gp *= (1 - Fg) * D * Gi * std::fabs(dh * hdi / in.z);
        }
        return dp + mp + gp + cp;
    }

    // Disney sample (disney.hlsli:233-380): returns direction, roughness (singular when 0), ok
    bool disney_sample(const Mat<R>& m, const V3<R>& in, const R rnd[3], V3<R>& dir, R& rough) const {
        R ax, ay; alphas(m, ax, ay);
        const R ac = (1 - m.clearcoat_gloss()) * R(0.1) + m.clearcoat_gloss() * R(0.001);
        const R metallic = m.metallic(), tr = m.transmission();
        const R dw = (1 - metallic) * (1 - tr), mw = (1 - tr * (1 - metallic)), gw = (1 - metallic) * tr, cw = m.clearcoat();
        auto reflect = [&](const V3<R>& h) { return normalize(-in + h * (2 * dot(in, h))); };
        if (in.z >= 0) {
            const R tw = dw + mw + gw + cw;
            const R dp = dw / tw, mp = mw / tw, gp = gw / tw;
            if (rnd[2] <= dp) { dir = sample_cos_hemisphere(rnd[0], rnd[1]); rough = 1; return true; }
            if (rnd[2] <= dp + mp) { dir = reflect(sample_vndf(in, ax, ay, rnd[0], rnd[1])); rough = m.roughness(); return true; }
            if (rnd[2] <= dp + mp + gp) {
                if (gp <= 0) { dir = V3<R>(0); rough = 0; return false; }
                V3<R> h = sample_vndf(in, ax, ay, rnd[0], rnd[1]);
                const R hdi = dot(h, in), eta = in.z > 0 ? m.eta1() : 1 / m.eta1();
                const R F = fresnel_dielectric(hdi, eta), u = (rnd[2] - (dp + mp)) / gp;
                if (u <= F) { dir = reflect(h); rough = 0; return true; }  // mRoughness left at 0 in the reference
                const R hdo2 = 1 - (1 - hdi * hdi) / (eta * eta);
                if (hdo2 <= 0) { dir = V3<R>(0); rough = 0; return false; }
                if (hdi < 0) h = -h;
                dir = -in / eta + h * (std::fabs(hdi) / eta - std::sqrt(hdo2));
                rough = m.roughness();
                return true;
            }
            const R a2 = ac * ac;
            const R ch = std::sqrt(std::max(R(0), (1 - std::pow(a2, 1 - rnd[0])) / (1 - a2)));
            const R sh = std::sqrt(std::max(1 - ch * ch, R(0))), az = 2 * PI<R>() * rnd[1];
            dir = reflect(V3<R>(sh * std::cos(az), sh * std::sin(az), ch));
            rough = std::sqrt(ac);
            return true;
        }
        V3<R> h = sample_vndf(in, ax, ay, rnd[0], rnd[1]);
        if (h.z < 0) h = -h;
        const R hdi = dot(h, in), eta = in.z > 0 ? m.eta1() : 1 / m.eta1();
        const R F = fresnel_dielectric(hdi, eta);
        if (rnd[2] <= F) { dir = reflect(h); rough = m.roughness(); return true; }
        const R hdo2 = 1 - (1 - hdi * hdi) / (eta * eta);
        if (hdo2 <= 0) { dir = V3<R>(0); rough = 0; return false; }
        if (hdi < 0) h = -h;
        dir = -in / eta + h * (std::fabs(hdi) / eta - std::sqrt(hdo2));
        rough = m.roughness();
        return true;
    }

    // evaluateReflectance: reflectance (f*cos), fwd pdf, rev pdf
    void eval(const Mat<R>& m, const V3<R>& in, const V3<R>& out, V3<R>& f, R& fwd, R& rev) const {
        if (lambert()) {  // lambertian.hlsli:16-27
            if (in.z * out.z < 0) { f = V3<R>(0); fwd = rev = 0; return; }
            f = m.base() * (std::fabs(out.z) / PI<R>());
            fwd = cos_hemisphere_pdfw(std::max(R(1e-5), std::fabs(out.z)));
            rev = cos_hemisphere_pdfw(std::max(R(1e-5), std::fabs(in.z)));
            return;
        }
        f = disney_eval(m, in, out);
        fwd = disney_pdf(m, in, out);
        rev = disney_pdf(m, out, in);
    }
    // sampleDirection: returns false on a failed sample (zero direction)
    bool sample_dir(const Mat<R>& m, const V3<R>& in, const R rnd[3], V3<R>& dir, V3<R>& f, R& fwd, R& rev, R& rough) const {
        if (lambert()) {  // lambertian.hlsli:29-38
            dir = sample_cos_hemisphere(rnd[0], rnd[1]);
            if (in.z < 0) dir = -dir;
            f = m.base() * (std::fabs(dir.z) / PI<R>());
            fwd = cos_hemisphere_pdfw(std::max(R(1e-5), std::fabs(dir.z)));
            rev = cos_hemisphere_pdfw(std::max(R(1e-5), std::fabs(in.z)));
            rough = 1;
            return true;
        }
        const bool ok = disney_sample(m, in, rnd, dir, rough);
        eval(m, in, dir, f, fwd, rev);
        return ok;
    }

    // ---------------------------------------------------------------- lights (lights.hlsli)
    R texel_lum(const Image<R>& im, uint32_t level, int x, int y) const {
        if (x < 0 || y < 0 || x >= (int)im.lw[level] || y >= (int)im.lh[level]) return 0;  // outside the level
        return im.lum[level][(size_t)y * im.lw[level] + x];
    }

    // SampleTexel (lights.hlsli:49-96)
    void sample_texel(const Image<R>& im, R rx, R ry, R& u, R& v, R& pdf) const {
        const uint32_t levels = (uint32_t)im.lum.size();
        pdf = 1;
        int cx = 0, cy = 0;
        uint32_t lx = 1, ly = 1;
        const uint32_t lim = std::min(11u, levels - 1);
        for (uint32_t i = 1; i < lim; ++i) {
            const uint32_t level = levels - 1 - i;
            const uint32_t ex = im.lw[level], ey = im.lh[level];
            const R inv_h = R(1) / (R)ey;
            cx *= (int)(ex / lx); cy *= (int)(ey / ly);
            R pp[4] = {0, 0, 0, 0};
            if ((int)ex - cx > 1) {
                const R sy = std::sin(PI<R>() * (cy + R(0.5)) * inv_h);
                pp[0] = texel_lum(im, level, cx, cy) * sy; pp[1] = texel_lum(im, level, cx + 1, cy) * sy;
            }
            if ((int)ey - cy > 1) {
                const R sy = std::sin(PI<R>() * (cy + R(1.5)) * inv_h);
                pp[2] = texel_lum(im, level, cx, cy + 1) * sy; pp[3] = texel_lum(im, level, cx + 1, cy + 1) * sy;
            }
            const R sum = pp[0] + pp[1] + pp[2] + pp[3];
            if (sum < R(1e-6)) continue;
            for (int j = 0; j < 4; ++j) pp[j] /= sum;
            for (int j = 0; j < 4; ++j) {
                if (j == 3 || rx < pp[j]) { cx += j % 2; cy += j / 2; pdf *= pp[j]; rx /= pp[j]; break; }
                rx -= pp[j];
            }
            lx = ex; ly = ey;
        }
        pdf *= (R)(lx * ly);
        u = ((R)cx + rx) / (R)lx;
        v = ((R)cy + ry) / (R)ly;
    }
    // SampleTexelPdf (lights.hlsli:97-138)
    R sample_texel_pdf(const Image<R>& im, R u, R v) const {
        const uint32_t levels = (uint32_t)im.lum.size();
        R pdf = 1;
        uint32_t lx = 1, ly = 1;
        const uint32_t lim = std::min(11u, levels - 1);
        for (uint32_t i = 1; i < lim; ++i) {
            const uint32_t level = levels - 1 - i;
            const uint32_t ex = im.lw[level], ey = im.lh[level];
            const R inv_h = R(1) / (R)ey;
            const int ux = (int)((R)ex * u), uy = (int)((R)ey * v);
            const int cx = (ux / 2) * 2, cy = (uy / 2) * 2;
            const int ox = std::min(ux - cx, 1), oy = std::min(uy - cy, 1);
            R pp[4] = {0, 0, 0, 0};
            if ((int)ex - cx > 1) {
                const R sy = std::sin(PI<R>() * (cy + R(0.5)) * inv_h);
                pp[0] = texel_lum(im, level, cx, cy) * sy; pp[1] = texel_lum(im, level, cx + 1, cy) * sy;
            }
            if ((int)ey - cy > 1) {
                const R sy = std::sin(PI<R>() * (cy + R(1.5)) * inv_h);
                pp[2] = texel_lum(im, level, cx, cy + 1) * sy; pp[3] = texel_lum(im, level, cx + 1, cy + 1) * sy;
            }
            const R sum = pp[0] + pp[1] + pp[2] + pp[3];
            if (sum < R(1e-6)) continue;
            pdf *= pp[oy * 2 + ox] / sum;
            lx = ex; ly = ey;
        }
        return pdf * (R)(lx * ly);
    }

    // EvaluateEnvironment (lights.hlsli:143-164)
    V3<R> eval_env(const V3<R>& dir, R& pdfw) const {
        pdfw = 0;
        if (!has_env()) return V3<R>(0);
        V3<R> e((R)s.f32(s.mat, s.env_addr), (R)s.f32(s.mat, s.env_addr + 4), (R)s.f32(s.mat, s.env_addr + 8));
        const uint32_t img = s.u32(s.mat, s.env_addr + 12);
        if (img < s.images.size()) {
            R u, v; cart_to_uv(dir, u, v);
            e = e * s.images[img].sample(u, v);
            pdfw = sample_texel_pdf(env_samp(img), u, v) / (2 * PI<R>() * PI<R>() * std::sqrt(1 - dir.y * dir.y));
        } else {
            pdfw = 1 / (4 * PI<R>());
        }
        if (light_count() > 0) pdfw *= (R)p.env_prob;
        return e;
    }

    // the luminance tables that drive environment sampling: the image's own, or its bilinear
    // footprint (S2_FLAG_ENV_FOOTPRINT_PDF, an extension of the reference's SampleTexel)
    const Image<R>& env_samp(uint32_t img) const {
        return (p.flags & S2_FLAG_ENV_FOOTPRINT_PDF) ? s.env_fp : s.images[img];
    }

    struct Illum {
        V3<R> radiance; R pdf; V3<R> dir; R dist; V3<R> pos; R cos_light; bool finite;
    };
    // SampleEmission + SampleIllumination (lights.hlsli:166-262)
    Illum sample_illum(const float rnd_in[4], const V3<R>& ref) const {
        Illum r{V3<R>(0), 0, V3<R>(0), 0, V3<R>(0), 0, true};
        R rnd[4] = {rnd_in[0], rnd_in[1], rnd_in[2], rnd_in[3]};
        const uint32_t L = light_count();
        if (has_env()) {
            if (L == 0 || rnd[3] < (R)p.env_prob) {
                const uint32_t img = s.u32(s.mat, s.env_addr + 12);
                V3<R> dir; R pdf;
                if (img < s.images.size()) {
                    R u, v; sample_texel(env_samp(img), rnd[0], rnd[1], u, v, pdf);
                    dir = uv_to_cart(u, v);
                    pdf /= (2 * PI<R>() * PI<R>() * std::sqrt(1 - pow2(dir.y)));
                } else {
                    dir = sample_uniform_sphere(rnd[0], rnd[1]);
                    pdf = 1 / (4 * PI<R>());
                }
                if (L > 0) pdf *= (R)p.env_prob;
                r.pdf = pdf; r.finite = false; r.dist = std::numeric_limits<R>::infinity(); r.cos_light = 1;
                r.dir = dir;
                R tmp; r.radiance = eval_env(dir, tmp);
                return r;
            }
            if (L > 0) rnd[3] = (rnd[3] - (R)p.env_prob) / (1 - (R)p.env_prob);
        }
        if (L == 0) return r;
        const uint32_t inst = s.light_map[(uint32_t)(rnd[2] * L) % L];
        R pdf = R(1) / (R)L;
        if (has_env()) pdf *= 1 - (R)p.env_prob;
        if ((s.inst_word0[inst] & 0xfu) != S2_INSTANCE_TYPE_MESH) return r;
        const uint32_t pc = s.prim_count[inst];
        const uint32_t prim = (uint32_t)(rnd[3] * pc) % pc;
        pdf /= (R)pc;
        const R a = std::sqrt(rnd[0]);
        const SD<R> sd = shading(inst, prim, 1 - a, a * rnd[1]);
        pdf /= sd.area;
        const Mat<R> m = material(sd.mat, sd.u, sd.v);
        r.radiance = m.emission();
        r.pos = sd.pos;
        r.dir = sd.pos - ref;
        r.dist = length(r.dir);
        r.dir = r.dir / r.dist;
        r.cos_light = -dot(sd.gn, r.dir);
        r.pdf = pdf;
        if (r.cos_light <= 0) { r.radiance = V3<R>(0); r.pdf = 0; }
        return r;
    }

    // LightSamplePdfA (lights.hlsli:264-272)
    R light_pdfa(uint32_t inst, R area) const {
        const uint32_t L = light_count();
        if (L == 0) return 0;
        R pdf = (R(1) / (R)s.prim_count[inst]) / (area * (R)L);
        if (has_env()) pdf *= 1 - (R)p.env_prob;
        return pdf;
    }

    bool occluded(const V3<R>& o, const V3<R>& d, R tmax) {
        shadow_rays++;
        return trace(s, o, d, R(0), tmax, true, !(p.flags & FLAG_NO_ALPHA)).hit;
    }

    // ---------------------------------------------------------------- camera path
    struct Out {
        R rad[3];
        float albedo[4];
        uint32_t vis[2];
        float depth[4];
        float prev_uv[2];
        uint32_t ids[2];
    };

    // one sample of one pixel (testrenderer.slang:938-1071 + :751-808)
    void render_sample(const S2View& view, int px, int py, uint32_t seed, Out& out) {
        out.rad[0] = out.rad[1] = out.rad[2] = 0;
        Rng rng((uint32_t)px, (uint32_t)py, seed, (p.flags & FLAG_PCG32) != 0);
        R offx = R(0.5), offy = R(0.5);
        if (p.flags & FLAG_PIXEL_JITTER) { float f[4]; rng.next_float(f); offx = f[0]; offy = f[1]; }
        // ViewData::toWorld (compat/scene.h:152-157) with ProjectionData::backProject (transform.h:159-170)
        const R W = (R)(view.image_max[0] - view.image_min[0]), H = (R)(view.image_max[1] - view.image_min[1]);
        const R uvx = ((R)px + offx - view.image_min[0]) / W, uvy = ((R)py + offy - view.image_min[1]) / H;
        const R cx = 2 * uvx - 1, cy = -(2 * uvy - 1);
        const R* pr = nullptr; (void)pr;
        const R sx = view.projection[0], sy = view.projection[1], ox = view.projection[2], oy = view.projection[3], nr = view.projection[4];
        const R sg = nr > 0 ? 1 : (nr < 0 ? -1 : 0);
        V3<R> ld;
        if (view.projection[7] < 0) { ld = V3<R>((cx - ox) / sx, (cy - oy) / sy, nr); }
        else ld = V3<R>(nr * (cx * sg - ox) / sx, nr * (cy * sg - oy) / sy, nr);
        ld = normalize(ld);
        R cam[12]; for (int k = 0; k < 12; ++k) cam[k] = (R)view.camera_to_world[k];
        V3<R> org(cam[3], cam[7], cam[11]);
        V3<R> dir = unpack_normal<R>(pack_normal(normalize(s.xvec(cam, ld))));
        V3<R> thr(1);
        uint32_t len = 0;
        R dir_pdf = 0;          // mDirPdfW (half)
        R isect_dist = 0;       // mIntersectionDistance (half)
        R isect_pdfa = 0;       // mIntersectionPdfA (half)
        const bool nee = !(p.flags & FLAG_NO_NEE);
        auto add = [&](const V3<R>& rad, R w, uint32_t path_len) {
            if (path_len < p.min_len) return;
            if (!(w > 0) || all_nonpos(rad)) return;
            out.rad[0] += rad.x * w; out.rad[1] += rad.y * w; out.rad[2] += rad.z * w;
        };
        while (len + 1 <= p.max_len) {
            // TraceRay (testrenderer.slang:1026-1058)
            ext_rays++;
            const Hit<R> h = trace(s, org, dir, R(0), std::numeric_limits<R>::infinity(), false, !(p.flags & FLAG_NO_ALPHA));
            len++;
            const uint32_t inst = h.hit ? s.tid[h.tri].inst : 0xffffffffu;
            const uint32_t prim = h.hit ? s.tid[h.tri].prim : 0xffffffffu;
            if (!h.hit) {
                isect_dist = std::numeric_limits<R>::infinity();
                if (len == 1) {
                    out.albedo[0] = out.albedo[1] = out.albedo[2] = out.albedo[3] = 1;
                    out.vis[0] = 0xffffffffu; out.vis[1] = pack_normal(dir);
                    out.depth[0] = out.depth[1] = std::numeric_limits<float>::infinity(); out.depth[2] = out.depth[3] = 1;
                    out.prev_uv[0] = (float)(((R)px + R(0.5)) / W); out.prev_uv[1] = (float)(((R)py + R(0.5)) / H);
                    out.ids[0] = out.ids[1] = 0xffffffffu;
                }
                R env_pdf;
                const V3<R> e = thr * eval_env(dir, env_pdf);
                if (any_pos(e)) {
                    R w = 1;
                    if (len > 1 && nee && dir_pdf > 0) {
                        const R light_pdf = (p.flags & FLAG_REF_ENV_MIS) ? (R(1) / PI<R>()) / pow2(s.sphere[3]) : env_pdf;
                        w = mis(dir_pdf, light_pdf);
                    }
                    add(e, w, len);
                }
                break;
            }
            SD<R> sd = shading(inst, prim, h.b1, h.b2);
            if (!(p.flags & FLAG_NO_NORMAL_MAPS)) normal_map(sd);
            isect_dist = (R)half_round((float)h.t);
            isect_pdfa = (R)half_round((float)light_pdfa(inst, sd.area));
            const Mat<R> m = material(sd.mat, sd.u, sd.v);
            // ProcessInteraction (testrenderer.slang:816-935)
            const V3<R> in = sd.to_local(-dir);
            const R cos_in = std::fabs(in.z);
            if (len == 1) {
                const V3<R> a = m.base();
                out.albedo[0] = (float)a.x; out.albedo[1] = (float)a.y; out.albedo[2] = (float)a.z; out.albedo[3] = 1;
                out.vis[0] = (inst & 0xffffu) | (prim << 16); out.vis[1] = sd.ns;
                out.ids[0] = inst; out.ids[1] = prim;
                // StoreAuxillaryData (testrenderer.slang:195-218)
                R pv[12]; for (int k = 0; k < 12; ++k) pv[k] = (R)view.prev_world_to_camera[k];
                const V3<R> pc = s.xpoint(pv, s.xpoint(&s.motion[12 * (size_t)inst], sd.pos));
                R ppx = (R)px + R(0.5), ppy = (R)py + R(0.5);
                const R nrp = view.projection[4];
                if ((pc.z > 0) == (nrp > 0) && pc.z != 0) {
                    const R x4 = pc.x * view.projection[0] + pc.z * view.projection[2];
                    const R y4 = pc.y * view.projection[1] + pc.z * view.projection[3];
                    const R z4 = std::fabs(nrp), w4 = pc.z * (nrp > 0 ? 1 : -1);
                    if (!(std::fabs(x4) >= std::fabs(w4) || std::fabs(y4) >= std::fabs(w4) || std::fabs(z4) >= std::fabs(w4))) {
                        ppx = view.image_min[0] + W * (x4 / w4 * R(0.5) + R(0.5));
                        ppy = view.image_min[1] + H * (-y4 / w4 * R(0.5) + R(0.5));
                    }
                }
                out.prev_uv[0] = (float)(ppx / W); out.prev_uv[1] = (float)(ppy / H);
                out.depth[0] = (float)isect_dist; out.depth[1] = (float)length(pc); out.depth[2] = out.depth[3] = 1;
            }
            if (in.z > 0) {
                const V3<R> e = thr * m.emission();
                if (any_pos(e)) {
                    R w = 1;
                    if (len > 1 && nee && dir_pdf > 0) w = mis(dir_pdf * (cos_in / pow2(isect_dist)), isect_pdfa);
                    add(e, w, len);
                }
            }
            if (len >= p.max_len) break;
            const Mat<R> ms = samp ? material(sd.mat, sd.u, sd.v, samp) : m;
            if (!can_eval(ms)) break;
            const bool sing = singular(ms);
            if (!sing && nee) connect_to_light(m, sd, in, thr, rng, len, add, inst, prim, samp ? &ms : nullptr);
            const R cp = std::min(R(1), cont_prob(ms));
            if (!(p.flags & FLAG_NO_RR)) {
                float f[4]; rng.next_float(f);
                if ((R)f[0] > cp) break;
            }
            float f[4]; rng.next_float(f);
            const R rnd3[3] = {f[0], f[1], f[2]};
            V3<R> sdir, refl; R fwd, rev, rough;
            sample_dir(ms, in, rnd3, sdir, refl, fwd, rev, rough);
            if (samp) { V3<R> fe; R a, b; eval(m, in, sdir, fe, a, b); refl = fe; }
            const R cpm = (p.flags & FLAG_NO_RR) ? R(1) : cp;
            fwd *= cpm; rev *= cpm;
            thr = thr * refl / fwd;
            dir_pdf = (rough == 0 || sing) ? R(0) : (R)half_round((float)fwd);
            thr = thr * sd.snc(in, sdir);
            const V3<R> wd = sd.to_world(sdir);
            dir = unpack_normal<R>(pack_normal(wd));
            org = ray_offset(sd.pos, sd.gn, wd);
            if (std::isnan(thr.x) || std::isnan(thr.y) || std::isnan(thr.z)) break;
            if (all_nonpos(thr)) break;
        }
    }

    // ReservoirSampleDataDI (testrenderer.slang:568-606): a light sample evaluated at one vertex
    struct DI {
        float x[4] = {0, 0, 0, 0};
        R src_pdf = 0, wtoa = 0, misw = 0, dist = 0;
        V3<R> contrib = V3<R>(0), dir = V3<R>(0);
        R vis = 1;  // visibility traced in the reuse-visibility mode
        R target() const { return luminance(contrib) * wtoa; }
    };
    DI eval_di(const Mat<R>& m, const SD<R>& sd, const V3<R>& in, const float x[4], R cp) const {
        DI c;
        for (int k = 0; k < 4; ++k) c.x[k] = x[k];
        const Illum r = sample_illum(x, sd.pos);
        c.src_pdf = r.pdf;
        if (luminance(r.radiance) > 0 && r.pdf > 0) {
            const V3<R> out = sd.to_local(r.dir);
            V3<R> f; R fwd, rev; eval(m, in, out, f, fwd, rev);
            f = f * sd.snc(in, out);
            fwd *= cp;
            c.contrib = f * r.radiance;
            c.wtoa = r.finite ? r.cos_light / pow2(r.dist) : R(1);
            const R AtoW = r.finite ? pow2(r.dist) / r.cos_light : R(1);
            c.misw = mis(r.pdf, fwd / AtoW);
            c.dir = r.dir; c.dist = r.dist;
        }
        return c;
    }

    // ReservoirReuse (testrenderer.slang:608-663): pairwise MIS between the current reservoir
    // and the stored one
    void reservoir_reuse(const Mat<R>& m, const SD<R>& sd, const V3<R>& in, R cp, const GridRecord<R>& q, DI& cur,
                         R& iw, R& M, Rng& rng, bool vis_on) {
        DI nw = eval_di(m, sd, in, q.rnd, cp);
        // gReSTIR_DI_Reuse_Visibility (testrenderer.slang:611-616): q's sample in the current domain
        // carries its visibility in the contribution; the target pdf stays unshadowed
        if (vis_on && nw.target() > 0 && occluded(ray_offset(sd.pos, sd.gn, nw.dir), nw.dir, adjust_distance(nw.dist)))
            nw.vis = 0;
        R phat_q = 0;
        {
            SD<R> sdq = shading_local(q.inst, q.prim, q.local_pos);
            if (!(p.flags & FLAG_NO_NORMAL_MAPS)) normal_map(sdq);
            const Mat<R> mq = material(sdq.mat, sdq.u, sdq.v);
            const R cpq = (p.flags & FLAG_NO_RR) ? R(1) : cont_prob(mq);
            const DI cq = eval_di(mq, sdq, q.dir_in, cur.x, cpq);
            if (cq.target() > 0) phat_q = cq.target();
        }
        const R m0 = mis(M * cur.target(), q.M * phat_q);
        const R m1 = mis(q.M * q.target, M * nw.target());
        const R w0 = m0 * cur.target() * iw, w1 = m1 * nw.target() * q.W;
        M += q.M;
        const R total = w0 + w1;
        float u[4]; rng.next_float(u);
        if ((R)u[0] * total <= w1) cur = nw;
        iw = cur.target() > 0 ? total / cur.target() : R(0);
    }

    template <class Add>
    void connect_to_light(const Mat<R>& m, const SD<R>& sd, const V3<R>& in, const V3<R>& thr, Rng& rng, uint32_t len,
                          Add& add, uint32_t inst, uint32_t prim, const Mat<R>* msamp = nullptr) {
        const R cp = (p.flags & FLAG_NO_RR) ? R(1) : cont_prob(msamp ? *msamp : m);
        if (p.flags & FLAG_RESTIR) {
            // SampleIlluminationReSTIR (testrenderer.slang:665-726) + ConnectToLight (:730-747)
            DI best; R wsum = 0;
            for (uint32_t i = 0; i < p.restir_m; ++i) {
                float x[4]; rng.next_float(x);
                const DI c = eval_di(m, sd, in, x, cp);
                if (c.target() <= 0) continue;
                const R risw = c.target() / c.src_pdf;
                wsum += risw;
                float u[4]; rng.next_float(u);
                if ((R)u[0] <= risw / wsum) best = c;
            }
            R iw = best.target() > 0 ? wsum / ((R)p.restir_m * best.target()) : R(0);
            // gReSTIR_DI_Reuse_Visibility (testrenderer.slang:689-694): canonical visibility first
            const bool vis_on = grid_cur && (p.flags & FLAG_RESTIR_REUSE_VIS);
            if (vis_on) {
                if (best.target() > 0 && occluded(ray_offset(sd.pos, sd.gn, best.dir), best.dir, adjust_distance(best.dist)))
                    best.vis = 0;
                if (!(best.vis > 0)) iw = 0;
            }
            if (grid_cur) {
                R M = (R)p.restir_m;
                if (grid_prev) {
                    float dr[4]; rng.next_float(dr);
                    R dx, dy; sample_concentric_disc<R>((R)dr[0], (R)dr[1], dx, dy);
                    const R csz = (R)grid_prev->cell_size(sd.pos);
                    const V3<R> qp = sd.pos + sd.to_world(V3<R>(dx * csz, dy * csz, 0));
                    const uint32_t cell = grid_prev->find(qp, grid_prev->cell_size(qp), false);
                    if (cell != 0xffffffffu && grid_prev->counter[cell] > 0) {
                        const uint32_t k = rng.next().x % grid_prev->counter[cell];
                        const GridRecord<R>& q = grid_prev->data[grid_prev->data_index[grid_prev->offset[cell] + k]];
                        reservoir_reuse(m, sd, in, cp, q, best, iw, M, rng, vis_on);
                    }
                }
                if (iw > 0) {
                    GridRecord<R> rec;
                    rec.local_pos = s.xpoint(&s.inv[12 * (size_t)inst], sd.pos);
                    rec.inst = inst; rec.prim = prim;
                    for (int k = 0; k < 4; ++k) rec.rnd[k] = best.x[k];
                    rec.target = best.target();
                    rec.W = iw;
                    rec.M = std::min(M, (R)p.max_m * (R)p.restir_m);
                    rec.dir_in = in;
                    grid_cur->append(sd.pos, rec);
                }
            }
            if (!(iw > 0)) return;
            iw *= best.wtoa;
            const V3<R> contrib = thr * best.contrib * (iw * best.vis);
            if (!(best.misw > 0) || all_nonpos(contrib)) return;
            if (len + 1 < p.min_len) return;
            const V3<R> o = ray_offset(sd.pos, sd.gn, best.dir);
            if (!vis_on && occluded(o, best.dir, adjust_distance(best.dist))) return;  // AddRadiance when traced
            add(contrib, best.misw, len + 1);
            return;
        }
        float x[4]; rng.next_float(x);
        const Illum r = sample_illum(x, sd.pos);
        if (all_nonpos(r.radiance) || r.pdf <= 0) return;
        const R AtoW = r.finite ? pow2(r.dist) / r.cos_light : R(1);
        const R dpw = r.pdf * AtoW;
        const V3<R> out = sd.to_local(r.dir);
        V3<R> f; R fwd, rev; eval(m, in, out, f, fwd, rev);
        if (msamp) { V3<R> fs; eval(*msamp, in, out, fs, fwd, rev); }
        f = f * sd.snc(in, out);
        fwd *= cp;
        const V3<R> contrib = thr * r.radiance * f / dpw;
        const R w = mis(r.pdf, fwd / AtoW);
        if (!(w > 0) || all_nonpos(contrib)) return;
        if (len + 1 < p.min_len) return;
        const V3<R> o = ray_offset(sd.pos, sd.gn, r.dir);
        if (occluded(o, r.dir, adjust_distance(r.dist))) return;
        add(contrib, w, len + 1);
    }
};

}  // namespace orc

// ============================================================================== C entry points
// The two ReSTIR reuse grids of one precision: the one the next call appends to and the previous.
template <class R> struct GridPair {
    std::unique_ptr<orc::CpuGrid<R>> g[2];
    int cur = 0;
    bool valid = false;
};

struct OracleScene {
    orc::Scene<double> d;
    orc::Scene<float> f;
    bool has_d = false, has_f = false;
    GridPair<double> grid_d;
    GridPair<float> grid_f;
    OracleScene* sampling = nullptr;  // detached-sampling scene (see Tracer::samp)
    const orc::Scene<double>* pick(const orc::Scene<double>&) const { return sampling ? &sampling->d : nullptr; }
    const orc::Scene<float>* pick(const orc::Scene<float>&) const { return sampling ? &sampling->f : nullptr; }
    GridPair<double>& grids(orc::Scene<double>&) { return grid_d; }
    GridPair<float>& grids(orc::Scene<float>&) { return grid_f; }
};

extern "C" {

// precision_mask: 1 = FP64 scene, 2 = FP32 scene (flattened with the GPU's float expression)
void* oracle_scene_create(const S2SceneDesc* desc, int precision_mask) {
    if (!desc) return nullptr;
    OracleScene* s = new OracleScene();
    if (precision_mask & 1) { s->d.load(desc, false); s->has_d = true; }
    if (precision_mask & 2) { s->f.load(desc, true); s->has_f = true; }
    return s;
}

void oracle_scene_destroy(void* s) { delete (OracleScene*)s; }

// rays: n x 8 floats (S2Ray).  Outputs t, instance, primitive, b1, b2 per ray.
int oracle_trace(void* sp, const float* rays, uint32_t n, int anyhit, int precision, double* t, uint32_t* inst,
                 uint32_t* prim, double* b1, double* b2, int threads) {
    OracleScene* s = (OracleScene*)sp;
    if (!s) return -1;
    if ((precision == 64 && !s->has_d) || (precision == 32 && !s->has_f)) return -1;
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const float* r = rays + 8 * i;
        if (precision == 64) {
            auto h = orc::trace<double>(s->d, orc::V3<double>(r[0], r[1], r[2]), orc::V3<double>(r[4], r[5], r[6]), r[3], r[7], anyhit != 0);
            t[i] = h.t; b1[i] = h.b1; b2[i] = h.b2;
            inst[i] = h.hit ? s->d.tid[h.tri].inst : 0xffffffffu; prim[i] = h.hit ? s->d.tid[h.tri].prim : 0xffffffffu;
        } else {
            auto h = orc::trace<float>(s->f, orc::V3<float>(r[0], r[1], r[2]), orc::V3<float>(r[4], r[5], r[6]), r[3], r[7], anyhit != 0);
            t[i] = h.t; b1[i] = h.b1; b2[i] = h.b2;
            inst[i] = h.hit ? s->f.tid[h.tri].inst : 0xffffffffu; prim[i] = h.hit ? s->f.tid[h.tri].prim : 0xffffffffu;
        }
    }
    return 0;
}

// Environment radiance (rgb) and its light-sampling solid-angle pdf for n directions (3 doubles
// each) under the flags of `rp` (FP64 scene): EvaluateEnvironment (lights.hlsli:143-164).
int oracle_env_eval(void* sp, const S2RenderParams* rp, const double* dirs, uint32_t n, double* rgb, double* pdf) {
    OracleScene* s = (OracleScene*)sp;
    if (!s || !rp || !s->has_d) return -1;
    orc::Params p{rp->min_path_length, rp->max_path_length, rp->spp, rp->frame_seed, rp->flags, 32u, rp->exposure,
                  rp->environment_sample_probability > 0 ? rp->environment_sample_probability : 0.9f};
    orc::Tracer<double> tr(s->d, p);
    for (uint32_t i = 0; i < n; ++i) {
        double pw = 0;
        const orc::V3<double> e = tr.eval_env(orc::V3<double>(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]), pw);
        rgb[3 * i] = e.x; rgb[3 * i + 1] = e.y; rgb[3 * i + 2] = e.z;
        pdf[i] = pw;
    }
    return 0;
}

// Renders pixels [x0,x1) x [y0,y1) (step `stride`) of `view` with `p.spp` samples each.
// sum/sumsq: W*H*3 doubles (pixel mean accumulators over samples, before exposure);
// aov buffers as in S2Aovs (may be null).  counters[0..1] += extension rays, shadow rays.
int oracle_render(void* sp, const S2View* view, const S2RenderParams* rp, int precision, int x0, int y0, int x1, int y1,
                  int stride, double* sum, double* sumsq, float* albedo, uint32_t* visibility, float* depth, float* prev_uv,
                  uint32_t* ids32, uint64_t* counters, int threads) {
    OracleScene* s = (OracleScene*)sp;
    if (!s || !view || !rp) return -1;
    const int W = view->image_max[0] - view->image_min[0];
    orc::Params p{rp->min_path_length, rp->max_path_length, rp->spp, rp->frame_seed, rp->flags,
                  rp->restir_candidates ? rp->restir_candidates : 32u, rp->exposure,
                  rp->environment_sample_probability > 0 ? rp->environment_sample_probability : 0.9f};
    if (stride < 1) stride = 1;
    std::vector<std::pair<int, int>> px;
    for (int y = y0; y < y1; y += stride) for (int x = x0; x < x1; x += stride) px.emplace_back(x, y);
    std::atomic<uint64_t> ext{0}, shd{0};
    const bool reuse = (rp->flags & orc::FLAG_RESTIR) && (rp->flags & orc::FLAG_RESTIR_REUSE);
    p.max_m = rp->restir_max_m > 0 ? rp->restir_max_m : 3.f;
    auto run = [&](auto& scene) {
        using R = std::remove_const_t<std::remove_reference_t<decltype(scene.tv[0])>>;
        auto& gp = s->grids(scene);
        orc::CpuGrid<R>* gcur = nullptr;
        orc::CpuGrid<R>* gprev = nullptr;
        if (reuse) {
            // TestRenderer.cpp:472-493: append to one grid, read the previous call's
            for (auto& g : gp.g) if (!g) g.reset(new orc::CpuGrid<R>());
            gcur = gp.g[gp.cur].get();
            gprev = gp.valid ? gp.g[gp.cur ^ 1].get() : nullptr;
            const uint64_t per = (uint64_t)px.size() * std::max(1u, std::min(2u, p.max_len ? p.max_len - 1 : 1u));
            gcur->clear(rp->restir_grid_cells ? rp->restir_grid_cells : 100000u,
                        (uint32_t)std::min<uint64_t>(per * p.spp, 1u << 24));
            gcur->min_cell = rp->restir_grid_cell_size > 0 ? rp->restir_grid_cell_size : 0.5f;
            gcur->pixel_radius = rp->restir_grid_pixel_radius;
            gcur->cam = orc::V3<R>(view->camera_to_world[3], view->camera_to_world[7], view->camera_to_world[11]);
            const int H = view->image_max[1] - view->image_min[1];
            gcur->dscale = std::tan(gcur->pixel_radius * view->projection[7] * std::max(1.f / (float)H, (float)H / ((float)W * (float)W)));
        } else {
            gp.valid = false;
        }
#pragma omp parallel num_threads(threads > 0 ? threads : omp_get_max_threads())
        {
            auto tr = orc::Tracer<R>(scene, p);
            tr.samp = s->pick(scene);
            tr.grid_cur = gcur;
            tr.grid_prev = gprev;
#pragma omp for schedule(dynamic, 16)
            for (int64_t k = 0; k < (int64_t)px.size(); ++k) {
                const int x = px[k].first, y = px[k].second;
                const size_t pi = (size_t)y * W + x;
                double acc[3] = {0, 0, 0}, acc2[3] = {0, 0, 0};
                for (uint32_t sidx = 0; sidx < p.spp; ++sidx) {
                    typename decltype(tr)::Out o{};
                    tr.render_sample(*view, x, y, p.seed + sidx, o);
                    for (int c = 0; c < 3; ++c) { acc[c] += (double)o.rad[c]; acc2[c] += (double)o.rad[c] * (double)o.rad[c]; }
                    if (sidx == 0) {
                        if (albedo) for (int c = 0; c < 4; ++c) albedo[4 * pi + c] = o.albedo[c];
                        if (visibility) { visibility[2 * pi] = o.vis[0]; visibility[2 * pi + 1] = o.vis[1]; }
                        if (depth) for (int c = 0; c < 4; ++c) depth[4 * pi + c] = o.depth[c];
                        if (prev_uv) { prev_uv[2 * pi] = o.prev_uv[0]; prev_uv[2 * pi + 1] = o.prev_uv[1]; }
                        if (ids32) { ids32[2 * pi] = o.ids[0]; ids32[2 * pi + 1] = o.ids[1]; }
                    }
                }
                if (sum) for (int c = 0; c < 3; ++c) sum[3 * pi + c] = acc[c];
                if (sumsq) for (int c = 0; c < 3; ++c) sumsq[3 * pi + c] = acc2[c];
            }
            ext += tr.ext_rays; shd += tr.shadow_rays;
        }
        if (reuse) {
            gcur->build();
            gp.cur ^= 1;
            gp.valid = true;
        }
    };
    if (precision == 64) { if (!s->has_d) return -1; run(s->d); }
    else { if (!s->has_f) return -1; run(s->f); }
    if (counters) { counters[0] += ext.load(); counters[1] += shd.load(); }
    return 0;
}

}  // extern "C"

// ---- the oracle's restatements of the reference's shader math, one function at a time, with the
// function ids and per-entry layouts of the reference build's ref_shader_math (oracle/ref_shader_math.cpp):
// 8 input and 9 output doubles per entry.  precision 32: the FP32 instantiation, else FP64.
template <class R> static void oracle_math_one(int fn, const double* a, double* o) {
    using V = orc::V3<R>;
    using T = orc::Tracer<R>;
    auto f = [&](int i) { return (R)a[i]; };
    auto u = [&](int i) { return (uint32_t)a[i]; };
    auto put3 = [&](const V& v, int at) { o[at] = (double)v.x; o[at + 1] = (double)v.y; o[at + 2] = (double)v.z; };
    switch (fn) {
        case 0: o[0] = orc::xxhash32(u(0)); break;
        case 1: o[0] = orc::pcg_hash(u(0)); break;
        case 2: { const orc::U4 r = orc::pcg4d({u(0), u(1), u(2), u(3)}); o[0] = r.x; o[1] = r.y; o[2] = r.z; o[3] = r.w; break; }
        case 3: {
            orc::Rng rng(u(0), u(1), u(2), false);
            rng.ctr = u(3);
            float r[4]; rng.next_float(r);
            for (int k = 0; k < 4; ++k) o[k] = r[k];
            break;
        }
        case 4: o[0] = orc::pack_normal(V(f(0), f(1), f(2))); break;
        case 5: put3(orc::unpack_normal<R>(u(0)), 0); break;
        case 6: o[0] = (double)T::GTR1(f(0), f(1)); break;
        case 7: o[0] = (double)T::GTR2(V(f(0), f(1), f(2)), f(3), f(4)); break;
        case 8: o[0] = (double)T::smith_gtr2(V(f(0), f(1), f(2)), f(3), f(4)); break;
        case 9: o[0] = (double)T::smith_gtr1(V(f(0), f(1), f(2))); break;
        case 10: put3(T::sample_vndf(V(f(0), f(1), f(2)), f(3), f(4), f(5), f(6)), 0); break;
        case 11: o[0] = (double)T::schlick(f(0), f(1)); break;
        case 12: o[0] = (double)T::fresnel_dielectric(f(0), f(1)); break;
        case 13: { R x, y; orc::sample_concentric_disc(f(0), f(1), x, y); o[0] = (double)x; o[1] = (double)y; break; }
        case 14: put3(orc::sample_cos_hemisphere(f(0), f(1)), 0); break;
        case 15: put3(orc::sample_uniform_sphere(f(0), f(1)), 0); break;
        case 16: { const R q = std::sqrt(f(0)); o[0] = (double)(1 - q); o[1] = (double)(q * f(1)); break; }
        case 17: {
            const V n(f(0), f(1), f(2));
            V t, b; orc::make_orthonormal(n, t, b);
            put3(t, 0); put3(b, 3); put3(n, 6);
            break;
        }
    }
}

extern "C" {

int oracle_math(int fn, const double* in, uint32_t n, double* out, int precision) {
    if (fn < 0 || fn > 17) return -1;
    for (uint32_t k = 0; k < n; ++k) {
        if (precision == 32) oracle_math_one<float>(fn, in + 8 * (size_t)k, out + 9 * (size_t)k);
        else oracle_math_one<double>(fn, in + 8 * (size_t)k, out + 9 * (size_t)k);
    }
    return 0;
}

// ---- unit-level entry points for known-answer tests (FP64)
void oracle_pcg4d(const uint32_t* in, uint32_t* out, uint32_t n) {
    for (uint32_t i = 0; i < n; ++i) {
        orc::U4 v = orc::pcg4d({in[4 * i], in[4 * i + 1], in[4 * i + 2], in[4 * i + 3]});
        out[4 * i] = v.x; out[4 * i + 1] = v.y; out[4 * i + 2] = v.z; out[4 * i + 3] = v.w;
    }
}
uint32_t oracle_pack_normal(double x, double y, double z) { return orc::pack_normal(orc::V3<double>(x, y, z)); }
void oracle_unpack_normal(uint32_t p, double* out) { auto v = orc::unpack_normal<double>(p); out[0] = v.x; out[1] = v.y; out[2] = v.z; }
float oracle_half_round(float x) { return orc::half_round(x); }

// BSDF evaluation on a packed material record (64 bytes): f (3), fwd, rev
void oracle_bsdf_eval(const uint32_t* mat_words, float emission_scale, int lambertian, const double* in, const double* out, double* res) {
    orc::Scene<double> dummy;
    orc::Params p{0, 5, 1, 0, lambertian ? orc::FLAG_LAMBERTIAN : 0u, 32, 0, 0.9f};
    orc::Tracer<double> tr(dummy, p);
    orc::Mat<double> m; for (int k = 0; k < 4; ++k) m.w[k] = mat_words[k]; m.escale = emission_scale;
    orc::V3<double> f; double fwd, rev;
    tr.eval(m, orc::V3<double>(in[0], in[1], in[2]), orc::V3<double>(out[0], out[1], out[2]), f, fwd, rev);
    res[0] = f.x; res[1] = f.y; res[2] = f.z; res[3] = fwd; res[4] = rev;
}
// BSDF sampling: dir (3), f (3), fwd, rev, roughness, ok
void oracle_bsdf_sample(const uint32_t* mat_words, int lambertian, const double* in, const double* rnd, double* res) {
    orc::Scene<double> dummy;
    orc::Params p{0, 5, 1, 0, lambertian ? orc::FLAG_LAMBERTIAN : 0u, 32, 0, 0.9f};
    orc::Tracer<double> tr(dummy, p);
    orc::Mat<double> m; for (int k = 0; k < 4; ++k) m.w[k] = mat_words[k]; m.escale = 0;
    orc::V3<double> d, f; double fwd, rev, rough;
    const bool ok = tr.sample_dir(m, orc::V3<double>(in[0], in[1], in[2]), rnd, d, f, fwd, rev, rough);
    res[0] = d.x; res[1] = d.y; res[2] = d.z; res[3] = f.x; res[4] = f.y; res[5] = f.z; res[6] = fwd; res[7] = rev; res[8] = rough; res[9] = ok;
}

}  // extern "C"

extern "C" {
uint32_t oracle_pcg_hash(uint32_t v) { return orc::pcg_hash(v); }
uint32_t oracle_xxhash32(uint32_t v) { return orc::xxhash32(v); }
}

extern "C" {
// Detached sampling for the adjoint checks: renders of `sp` take sampling decisions from `samp`
// (a scene with the same geometry and other images); NULL restores the normal mode.
void oracle_scene_set_sampling(void* sp, void* samp) { ((OracleScene*)sp)->sampling = (OracleScene*)samp; }
}
